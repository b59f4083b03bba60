"""ctypes wrapper of the reference itself (oracle/_ref/libwloopref_<size>.so).

The reference's modules/{lnk,smear,wloop} compiled unchanged from their
sources against a one-process openQCD-1.4 interface (oracle/refshim,
oracle/Makefile `ref`); openQCD fixes the lattice size at compile time, so
there is one library per size.  Test infrastructure: used by tests/ and by
bench.py's reference leg only, as the checker and the timed reference.

Each library holds its own gauge field (openQCD's udfld()) and module state;
the calls below mirror the reference's entry points on that field.
"""
import ctypes as C
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFDIR = os.path.join(ROOT, "oracle", "_ref")
_libs = {}

dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)


def so_path(n):
    return os.path.join(REFDIR, "libwloopref_%dx%dx%dx%d.so" % tuple(n))


def available(n) -> bool:
    return os.path.exists(so_path(n))


def sizes():
    """Lattice sizes (N0, N1, N2, N3) with a built reference library."""
    out = []
    if os.path.isdir(REFDIR):
        for f in sorted(os.listdir(REFDIR)):
            if f.startswith("libwloopref_") and f.endswith(".so"):
                out.append(tuple(int(x) for x in f[len("libwloopref_"):-3].split("x")))
    return out


class Ref:
    """The reference built for one lattice size."""

    def __init__(self, n):
        n = tuple(int(x) for x in n)
        if n not in _libs:
            L = C.CDLL(so_path(n))
            L.wlref_dims.argtypes = [ip]
            L.wlref_set_field.argtypes = [C.c_int, dp]
            L.wlref_get_field.argtypes = [dp]
            L.wlref_hyp.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int]
            L.wlref_ape.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.c_int]
            L.wlref_hyp_spatial.argtypes = [C.c_double, C.c_double, C.c_int, C.c_int, C.c_int]
            L.wlref_plaq_sum.restype = C.c_double
            L.wlref_project.argtypes = [dp, C.c_int]
            for f in (L.wlref_wloop_sum, L.wlref_measure):
                f.argtypes = [C.c_int, ip, C.c_int, C.c_int, C.c_int, dp, C.c_double, dp, C.c_int,
                              dp]
                f.restype = C.c_int
            dims = (C.c_int * 4)()
            self_max = L.wlref_dims(dims)
            if tuple(dims) != n:
                raise RuntimeError(f"{so_path(n)} was built for {tuple(dims)}")
            _libs[n] = (L, self_max)
        self.n = n
        self.lib, self.max_levels = _libs[n]
        self.volume = int(np.prod(n))

    # --- the gauge field (udfld) in the lexicographic su3_dble layout ------
    def set_field(self, bc: int, u: np.ndarray) -> None:
        u = np.ascontiguousarray(u, dtype=np.complex128)
        assert u.size == self.volume * 4 * 9
        self.lib.wlref_set_field(bc, u.ctypes.data_as(dp))

    def get_field(self) -> np.ndarray:
        u = np.empty((self.volume, 4, 3, 3), dtype=np.complex128)
        self.lib.wlref_get_field(u.ctypes.data_as(dp))
        return u

    # --- the reference's entry points on that field -------------------------
    def hyp_links(self, a1, a2, a3, proj=1, piter=4, which=0):
        """which 0: hyp_links, 1: hyp_time_links, 2: hyp_space_links"""
        self.lib.wlref_hyp(which, a1, a2, a3, proj, piter)

    def ape_links(self, alpha, proj=1, piter=4, time=0, nsweeps=1):
        self.lib.wlref_ape(alpha, proj, piter, time, nsweeps)

    def hyp_spatial_links(self, a1, a2, proj=1, piter=4, nsweeps=1):
        self.lib.wlref_hyp_spatial(a1, a2, proj, piter, nsweeps)

    def plaq_sum(self) -> float:
        return self.lib.wlref_plaq_sum()

    def project(self, m: np.ndarray, iterations: int) -> np.ndarray:
        m = np.ascontiguousarray(m, dtype=np.complex128).copy()
        flat = m.reshape(-1, 3, 3)
        for j in range(flat.shape[0]):
            self.lib.wlref_project(flat[j].ctypes.data_as(dp), iterations)
        return m

    def _loops(self, fn, p):
        if p.msl > self.max_levels:
            raise ValueError(f"msl {p.msl} > MAX_SM_LEVELS {self.max_levels} of this library")
        wl = np.empty(p.msl * p.msl * p.mwlt * p.mwlr * self.n[0])
        nss = (C.c_int * p.msl)(*[int(x) for x in p.nss[:p.msl]])
        aa = (C.c_double * 3)(*p.alpha_action)
        ah = (C.c_double * 2)(*p.alpha_hyp)
        k = fn(p.msl, nss, p.mwlt, p.mwlr, int(p.op_smear), aa, p.alpha_ape, ah, p.proj_iter,
               wl.ctypes.data_as(dp))
        assert k == wl.size
        return wl

    def wloop_sum(self, p) -> np.ndarray:
        """set_wloop_parms + wloop_sum on the current field (no action smearing)."""
        return self._loops(self.lib.wlref_wloop_sum, p)

    def measure(self, p) -> np.ndarray:
        """ms10's per-configuration work (main/ms10.c:633-646): hyp_links with
        alpha_action, then wloop_sum; the field is left HYP-smeared."""
        return self._loops(self.lib.wlref_measure, p)


def generate_links(n, bc, seed, eps):
    """The synthetic field from the oracle's copy of the generator (no
    product library involved)."""
    from tests import oracle as O
    return O.generate_links(n, bc, seed, eps)
