"""ctypes wrapper of the FP64 CPU oracle (oracle/_build/liboracle.so).

Test infrastructure: used by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py only, as the checker.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SO = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SO):
            import subprocess
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                           capture_output=True)
        L = C.CDLL(SO)
        dp, ip, i, d = C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_int, C.c_double
        L.orc_project.argtypes = [dp, i]
        L.orc_staple_sum.argtypes = [ip, dp, dp, i, i, dp]
        L.orc_hyp_links.argtypes = [ip, i, dp, d, d, d, i, i, i, i]
        L.orc_ape_links.argtypes = [ip, dp, d, i, i, i]
        L.orc_hyp_spatial_links.argtypes = [ip, dp, d, d, i, i]
        L.orc_plaq_sum.argtypes = [ip, i, dp]
        L.orc_plaq_sum.restype = d
        L.orc_wloop_sum.argtypes = [ip, i, dp, i, ip, i, i, i, d, dp, i, dp, dp, dp, dp]
        L.orc_wloop_sum.restype = i
        L.orc_set_threads.argtypes = [i]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _i(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _n(n):
    return np.asarray(n, dtype=np.int32)


def set_threads(k):
    lib().orc_set_threads(int(k))


def project(m, iterations):
    m = np.ascontiguousarray(m, dtype=np.complex128).copy()
    flat = m.reshape(-1, 3, 3)
    for j in range(flat.shape[0]):
        lib().orc_project(_d(flat[j].view(np.float64)), iterations)
    return m


def staple_sum(n, u1, u2, mu, nu, vb):
    vb = np.ascontiguousarray(vb, dtype=np.complex128).copy()
    nn = _n(n)
    lib().orc_staple_sum(_i(nn), _d(np.ascontiguousarray(u1).view(np.float64)),
                         _d(np.ascontiguousarray(u2).view(np.float64)), mu, nu,
                         _d(vb.view(np.float64)))
    return vb


def hyp_links(n, bc, u, a1, a2, a3, proj, piter, time=1, space=1):
    u = np.ascontiguousarray(u, dtype=np.complex128).copy()
    nn = _n(n)
    lib().orc_hyp_links(_i(nn), bc, _d(u.view(np.float64)), a1, a2, a3, proj, piter, time, space)
    return u


def ape_links(n, u, alpha, proj, piter, time=1, nsweeps=1):
    u = np.ascontiguousarray(u, dtype=np.complex128).copy()
    nn = _n(n)
    for _ in range(nsweeps):
        lib().orc_ape_links(_i(nn), _d(u.view(np.float64)), alpha, proj, piter, time)
    return u


def hyp_spatial_links(n, u, a1, a2, proj, piter, nsweeps=1):
    u = np.ascontiguousarray(u, dtype=np.complex128).copy()
    nn = _n(n)
    for _ in range(nsweeps):
        lib().orc_hyp_spatial_links(_i(nn), _d(u.view(np.float64)), a1, a2, proj, piter)
    return u


def plaq_sum(n, bc, u):
    nn = _n(n)
    return lib().orc_plaq_sum(_i(nn), bc, _d(np.ascontiguousarray(u).view(np.float64)))


def wloop_sum(n, bc, u, p, want_abs=False, want_plaq=False, want_levels=False):
    """Reference-algorithm wloop_sum on a HYP-smeared field u; p is a WloopParms."""
    nn = _n(n)
    vol = int(np.prod(n))
    wls = p.msl * p.msl * p.mwlt * p.mwlr * n[0]
    wl = np.empty(wls)
    wa = np.empty(wls) if want_abs else None
    pl = np.empty(p.msl) if want_plaq else None
    lv = np.empty((p.msl, vol, 3, 3, 3), dtype=np.complex128) if want_levels else None
    nss = np.zeros(8, dtype=np.int32)
    nss[:p.msl] = p.nss[:p.msl]
    ah = np.asarray(p.alpha_hyp, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.complex128)
    rc = lib().orc_wloop_sum(_i(nn), bc, _d(u.view(np.float64)), p.msl, _i(nss), p.mwlt, p.mwlr,
                             int(p.op_smear), p.alpha_ape, _d(ah), p.proj_iter, _d(wl),
                             _d(wa) if wa is not None else None,
                             _d(pl) if pl is not None else None,
                             _d(lv.view(np.float64)) if lv is not None else None)
    if rc != 0:
        raise ValueError("oracle rejected the parameters")
    out = [wl]
    if want_abs:
        out.append(wa)
    if want_plaq:
        out.append(pl)
    if want_levels:
        out.append(lv)
    return out[0] if len(out) == 1 else tuple(out)


def generate_links(n, bc, seed, eps):
    """The synthetic gauge field from oracle/fieldgen.c, the test-side copy of
    the product's generator (same bytes; checked in tests/test_reference.py)."""
    L = lib()
    if not getattr(L, "_gen_typed", False):
        L.orc_generate_links.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_uint64, C.c_double,
                                         C.POINTER(C.c_double)]
        L.orc_aux_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_uint32]
        L.orc_aux_uniform.restype = C.c_double
        L._gen_typed = True
    vol = int(np.prod(n))
    u = np.empty((vol, 4, 3, 3), dtype=np.complex128)
    nn = _n(n)
    L.orc_generate_links(_i(nn), int(bc), int(seed), float(eps), _d(u.view(np.float64)))
    return u


def aux_uniform(seed, index, tag):
    generate_links((1, 1, 1, 1), 3, 0, 0.0)  # binds the argument types
    return lib().orc_aux_uniform(int(seed), int(index), int(tag))
