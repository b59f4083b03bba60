"""wlg_plaq_sum_noalloc: the plaquette sum for callers that cannot allocate
device memory (their memory belongs to another allocator or a preallocated
arena, or cudaMalloc's device synchronisation is not acceptable where they
call).  It must agree with the ordinary entry point (wlg_plaq_sum) on the
same field, on consecutive calls (the shared scratch keeps the previous
call's contents), and reject lattices beyond its fixed scratch.

Collected last on purpose (file name), so a run that stops at the first
failure has run every other test before this one.  The test itself allocates
the device buffers (through torch); the entry point allocates nothing.
"""
import ctypes as C

import numpy as np
import pytest

from wloop_b200 import Context, generate_links
from wloop_b200._native import lib

pytestmark = pytest.mark.gpu

lib.wlg_plaq_sum_noalloc.restype = C.c_int
lib.wlg_plaq_sum_noalloc.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_void_p,
                                     C.c_void_p]


def _call(links_ptr, n, bc, out_ptr):
    nn = (C.c_int * 4)(*n)
    return lib.wlg_plaq_sum_noalloc(links_ptr, nn, bc, out_ptr, None)


# 1920 and 1536 sites fit one 2048-site chunk; 4096 and 8192 sites need two
# and four chunk partials and the strided sum over them
@pytest.mark.parametrize("n,bc", [((8, 6, 4, 10), 0), ((6, 8, 8, 4), 3), ((8, 8, 8, 8), 0),
                                  ((16, 8, 8, 8), 3)])
def test_noalloc_matches_plaq_sum_on_consecutive_calls(n, bc):
    import torch
    u = generate_links(n, bc, 4242, 0.3)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        ref = c.lnk_plaq_sum()
    links = torch.from_numpy(u.view(np.float64).reshape(-1).copy()).cuda()
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        assert _call(links.data_ptr(), n, bc, out.data_ptr()) == 0, lib.wlg_last_error()
        torch.cuda.synchronize()
        got = float(out.item())
        assert abs(got - ref) <= 1e-13 * abs(ref), (got, ref)


def test_noalloc_rejects_oversize_and_host_memory():
    import torch
    links = torch.zeros(64, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    assert _call(links.data_ptr(), (130, 64, 64, 64), 3, out.data_ptr()) == -1
    assert b"exceed the maximum" in lib.wlg_last_error()
    host = np.zeros(4 * 256 * 18)
    assert _call(host.ctypes.data, (4, 4, 4, 4), 3, out.data_ptr()) == -1
    assert b"device" in lib.wlg_last_error() or b"CUDA pointer" in lib.wlg_last_error()


def test_noalloc_smaller_lattice_after_larger_one():
    """The shared scratch keeps a larger call's partials; a smaller call that
    follows must read only the partials it wrote itself."""
    import torch
    out = torch.empty(1, dtype=torch.float64, device="cuda")
    res = {}
    for n, bc in (((16, 8, 8, 8), 3), ((8, 6, 4, 10), 3)):
        u = generate_links(n, bc, 77, 0.3)
        with Context(n, bc, "fp64") as c:
            c.upload(u)
            ref = c.lnk_plaq_sum()
        links = torch.from_numpy(u.view(np.float64).reshape(-1).copy()).cuda()
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        assert _call(links.data_ptr(), n, bc, out.data_ptr()) == 0, lib.wlg_last_error()
        torch.cuda.synchronize()
        res[n] = (float(out.item()), ref)
    for got, ref in res.values():
        assert abs(got - ref) <= 1e-13 * abs(ref), (got, ref)


def test_noalloc_rejects_memory_of_another_gpu():
    """A field on another GPU than the current one is refused before any
    launch (the kernel would read peer memory without peer access)."""
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    links = torch.zeros(4 * 256 * 18, dtype=torch.float64, device="cuda:1")
    out = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    torch.cuda.set_device(0)
    assert _call(links.data_ptr(), (4, 4, 4, 4), 3, out.data_ptr()) == -1
    assert b"lives on device 1" in lib.wlg_last_error()
