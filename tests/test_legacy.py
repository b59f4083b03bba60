"""The reference's own entry points (include/wloop_b200_legacy.h) served by
libwloop_b200.so.

CPU: parameter database and range checks (wloop_parms.c:96-194), the .par
record (wloop_parms.c:343-429), wl_idx, openQCD link addressing (lnk, lnkf,
lnk_plaq: lnkcom.c:840-896) and attach validation.
GPU: a C program written against the reference API (tests/legacy/check_unit.c,
the unit-field check of devel/wloop/check1.c) and HYP / plaquette through the
legacy names compared with the context API.
"""
import ctypes as C
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "wloop_b200", "_lib")
SCRIPT = r'''
import ctypes as C, sys, numpy as np
lib = C.CDLL(sys.argv[1])
'''


def _run_py(body):
    """Runs body in a fresh interpreter (the legacy layer is process-global)."""
    code = "import ctypes as C, numpy as np, sys\n" \
           f"lib = C.CDLL({os.path.join(LIBDIR, 'libwloop_b200.so')!r})\n" + body
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300)
    return r


ATTACH = r'''
n = (8, 4, 4, 6)
V = 8 * 4 * 4 * 6
x = np.indices(n).reshape(4, -1)
par = x.sum(axis=0) % 2
ipt = np.empty(V, dtype=np.int32)
ev = np.nonzero(par == 0)[0]; od = np.nonzero(par == 1)[0]
ipt[ev] = np.arange(len(ev)); ipt[od] = len(ev) + np.arange(len(od))
ud = np.zeros((4 * V, 18))
UDF = C.CFUNCTYPE(C.c_void_p)
udf = UDF(lambda: ud.ctypes.data)
nn = (C.c_int * 4)(*n)
lib.wloop_b200_attach(nn, BC, ipt.ctypes.data_as(C.POINTER(C.c_int)), udf)
'''


PARMS = r'''
class P(C.Structure):
    _fields_ = [("msl", C.c_int), ("nss", C.c_int * 8), ("mwlt", C.c_int), ("mwlr", C.c_int),
                ("wls", C.c_int), ("op_smear", C.c_int), ("alpha_action", C.c_double * 3),
                ("alpha_ape", C.c_double), ("alpha_hyp", C.c_double * 2), ("proj", C.c_int),
                ("proj_iter", C.c_int), ("wl_mat", C.POINTER(C.c_double))]
lib.set_wloop_parms.restype = P
lib.wloop_parms.restype = P
'''


def test_parms_and_par_record(tmp_path):
    body = ATTACH.replace("BC", "3") + PARMS + r'''
nss = (C.c_int * 8)(0, 5, 5, 5)
aa = (C.c_double * 3)(1.0, 1.0, 0.5)
ah = (C.c_double * 2)(0.0, 0.0)
p = lib.set_wloop_parms(4, nss, 4, 3, 0, aa, C.c_double(0.5), ah, 4)
assert p.msl == 4 and p.mwlt == 4 and p.mwlr == 3 and p.proj == 1 and p.proj_iter == 4
assert p.wls == 4 * 4 * 4 * 3 * 8
assert all(p.wl_mat[i] == 1.0 for i in range(p.wls))          # wloop_parms.c:188-189
assert lib.wl_idx(1, 2, 3, 2, 5) == 1 + 4 * (2 + 4 * (3 + 4 * (2 + 3 * 5)))
libc = C.CDLL(None)
libc.fopen.restype = C.c_void_p
libc.fopen.argtypes = [C.c_char_p, C.c_char_p]
libc.fclose.argtypes = [C.c_void_p]
lib.write_wloop_parms.argtypes = [C.c_void_p]
lib.check_wloop_parms.argtypes = [C.c_void_p]
f = libc.fopen(sys.argv[1].encode(), b"wb"); lib.write_wloop_parms(f); libc.fclose(f)
f = libc.fopen(sys.argv[1].encode(), b"rb"); lib.check_wloop_parms(f); libc.fclose(f)
print("ok")
'''
    par = str(tmp_path / "x.par")
    code = "import ctypes as C, numpy as np, sys\n" \
           f"lib = C.CDLL({os.path.join(LIBDIR, 'libwloop_b200.so')!r})\n" + body
    r = subprocess.run([sys.executable, "-c", code, par], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr
    raw = open(par, "rb").read()
    # (msl+4) int32 {nss, mwlt, mwlr, op_smear, proj_iter} + 6 doubles (wloop_parms.c:357-378)
    ints = struct.unpack("<8i", raw[:32])
    dbl = struct.unpack("<6d", raw[32:])
    assert ints == (0, 5, 5, 5, 4, 3, 0, 4)
    assert dbl == (0.5, 0.0, 0.0, 1.0, 1.0, 0.5)


def test_parms_range_errors_are_fatal():
    body = ATTACH.replace("BC", "3") + PARMS + r'''
nss = (C.c_int * 8)(0, 5, 5, 5)
aa = (C.c_double * 3)(1.0, 1.0, 0.5); ah = (C.c_double * 2)(0.0, 0.0)
lib.set_wloop_parms(4, nss, 6, 3, 0, aa, C.c_double(0.5), ah, 4)   # mwlt > N0/2+1
'''
    r = _run_py(body)
    assert r.returncode == 1 and "max wloop time extension out of range" in r.stderr


def test_lnk_addressing():
    """lnk/lnkf/lnk_plaq follow ofs_lnk (lnkcom.c:840-859): links live at odd points."""
    body = ATTACH.replace("BC", "3") + r'''
lib.lnk.restype = C.c_void_p
lib.lnk.argtypes = [C.c_void_p, C.c_int, C.c_int]
base = ud.ctypes.data
seen = set()
st = [4 * 4 * 6, 4 * 6, 6, 1]
for s in range(V):
    xs = np.unravel_index(s, n)
    for mu in range(4):
        off = (lib.lnk(base, int(ipt[s]), mu) - base) // 144
        iq = ipt[s]
        if iq >= V // 2:
            assert off == 8 * (iq - V // 2) + 2 * mu
        else:
            y = list(xs); y[mu] = (y[mu] + 1) % n[mu]
            iy = ipt[np.ravel_multi_index(y, n)]
            assert iy >= V // 2 and off == 8 * (iy - V // 2) + 2 * mu + 1
        seen.add(off)
assert seen == set(range(4 * V))
print("ok")
'''
    r = _run_py(body)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr


def test_attach_rejects_bad_ipt():
    body = r'''
ipt = np.zeros(8 * 4 * 4 * 6, dtype=np.int32)
UDF = C.CFUNCTYPE(C.c_void_p); udf = UDF(lambda: 0)
lib.wloop_b200_attach((C.c_int * 4)(8, 4, 4, 6), 3, ipt.ctypes.data_as(C.POINTER(C.c_int)), udf)
'''
    r = _run_py(body)
    assert r.returncode == 1 and "ipt is not a permutation" in r.stderr


def _build_check_unit(tmp):
    exe = os.path.join(tmp, "check_unit")
    subprocess.run(["/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc", "-O2",
                    "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "legacy", "check_unit.c"), "-o", exe,
                    "-L", LIBDIR, "-lwloop_b200", "-Wl,-rpath," + LIBDIR, "-lm"], check=True)
    return exe


def test_check_unit_program_builds(tmp_path):
    assert os.path.exists(_build_check_unit(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("bc", [0, 3])
def test_check_unit_program(tmp_path, bc):
    exe = _build_check_unit(str(tmp_path))
    with open(os.path.join(ROOT, "tests", "legacy", "unit.in")) as fin:
        r = subprocess.run([exe, str(bc)], stdin=fin, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "unit field check: ok" in r.stdout
    assert "msl = 4" in r.stdout and "alpha = 0.5" in r.stdout


@pytest.mark.gpu
def test_legacy_hyp_and_plaquette_match_context():
    body = ATTACH.replace("BC", "0") + r'''
sys.path.insert(0, %r)
from wloop_b200 import Context, generate_links
u = generate_links(n, 0, 77, 0.3)
# pack into the openQCD layout through lnk()
lib.lnk.restype = C.c_void_p
lib.lnk.argtypes = [C.c_void_p, C.c_int, C.c_int]
base = ud.ctypes.data
for s in range(V):
    for mu in range(4):
        off = (lib.lnk(base, int(ipt[s]), mu) - base) // 144
        ud[off] = u[s, mu].view(np.float64).reshape(18)
lib.lnk_plaq_sum.restype = C.c_double
lib.lnk_plaq_sum.argtypes = [C.c_void_p]
p0 = lib.lnk_plaq_sum(C.c_void_p(base))
lib.hyp_links.argtypes = [C.c_double] * 3 + [C.c_int] * 3
lib.hyp_links(1.0, 1.0, 0.5, 1, 4, 0)
with Context(n, 0, "fp64") as c:
    c.upload(u)
    q0 = c.lnk_plaq_sum()
    c.hyp_links(1.0, 1.0, 0.5, 1, 4)
    ref = c.download()
got = np.empty_like(ref)
for s in range(V):
    for mu in range(4):
        off = (lib.lnk(base, int(ipt[s]), mu) - base) // 144
        got[s, mu] = ud[off].view(np.complex128).reshape(3, 3)
assert abs(p0 - q0) < 1e-12 * abs(q0)
assert np.array_equal(got, ref)
print("ok")
''' % ROOT
    r = _run_py(body)
    assert r.returncode == 0 and "ok" in r.stdout, r.stdout + r.stderr
