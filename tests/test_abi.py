"""The C ABI: libwloop_b200.so loads without a GPU and exports every function
declared in include/*.h (no compute calls here)."""
import ctypes as C
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "wloop_b200", "_lib", "libwloop_b200.so")


def declared(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    text = re.sub(r"#[^\n]*", " ", text)
    text = re.sub(r"typedef[^;]*;", " ", text, flags=re.S)
    names = set()
    for stmt in text.split(";"):
        stmt = " ".join(stmt.split())
        m = re.match(r"^(?:extern \"C\" \{ )?(?:[A-Za-z_][\w ]*[\w\*]+\s*\**\s*)\b([A-Za-z_]\w*)\s*\(", stmt)
        if m and not stmt.startswith(("struct", "enum")):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(LIB)
    headers = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
               if f.endswith(".h")]
    names = set()
    for h in headers:
        names |= declared(h)
    assert len(names) > 80
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_library_loads_without_gpu_and_reports_errors():
    lib = C.CDLL(LIB)
    lib.wlg_last_error.restype = C.c_char_p
    lib.wlg_version.restype = C.c_int
    assert lib.wlg_version() >= 100
    h = C.c_void_p()
    n = (C.c_int * 4)(4, 4, 4, 4)
    # bad boundary condition is rejected before any device call
    assert lib.wlg_create(n, 1, 0, 0, C.byref(h)) == -1
    assert b"boundary" in lib.wlg_last_error()
