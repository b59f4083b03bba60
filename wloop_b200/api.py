"""Host-side mirror of the wloop measurement interface over the C ABI.

The method names follow the reference's C entry points (include/smear.h,
include/lnk.h, include/wloop.h of bjoern-leder/wloop) so tests and drivers
read like the reference's own checks; every method runs on the GPU through
libwloop_b200.so.

Link fields on the host are numpy complex128 arrays of shape (V, 4, 3, 3)
(lexicographic sites x3 + N3*(x2 + N2*(x1 + N1*x0)), su3_dble byte layout).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from ._native import (WLG_FP64, WLG_MAX_SM_LEVELS, WLG_MIXED, WLG_OP_APE, WLG_OP_HYP, WlgError,
                      WlgParms, WlgRequest, check, dptr, iptr, lib)

APE, HYP = WLG_OP_APE, WLG_OP_HYP
PRECISIONS = {"fp64": WLG_FP64, "mixed": WLG_MIXED}


@dataclass
class WloopParms:
    """Mirror of wloop_parms_t (include/wloop.h:24-36); see set_wloop_parms."""
    msl: int
    nss: List[int]
    mwlt: int
    mwlr: int
    op_smear: int = APE
    alpha_action: Sequence[float] = (1.0, 1.0, 0.5)
    alpha_ape: float = 0.5
    alpha_hyp: Sequence[float] = (0.0, 0.0)
    proj_iter: int = 4

    @property
    def proj(self) -> int:  # wloop_parms.c:171
        return int(self.proj_iter > 0)

    def wls(self, n0: int) -> int:  # wloop_parms.c:182
        return self.msl * self.msl * self.mwlt * self.mwlr * n0

    def to_c(self) -> WlgParms:
        p = WlgParms()
        p.msl = self.msl
        for k in range(WLG_MAX_SM_LEVELS):
            p.nss[k] = int(self.nss[k]) if k < len(self.nss) else 0
        p.mwlt, p.mwlr, p.op_smear = self.mwlt, self.mwlr, int(self.op_smear)
        for k in range(3):
            p.alpha_action[k] = float(self.alpha_action[k])
        p.alpha_ape = float(self.alpha_ape)
        p.alpha_hyp[0], p.alpha_hyp[1] = float(self.alpha_hyp[0]), float(self.alpha_hyp[1])
        p.proj_iter = self.proj_iter
        return p


def set_wloop_parms(msl, nss, mwlt, mwlr, op_smear, alpha_action, alpha_ape, alpha_hyp,
                    proj_iter) -> WloopParms:
    """set_wloop_parms (wloop_parms.c:96-194); ranges are checked at use."""
    if op_smear not in (APE, HYP):
        raise WlgError("Unknown type of operator smearing")
    if msl < 1 or msl > WLG_MAX_SM_LEVELS:
        raise WlgError("max smearing level out of range")
    return WloopParms(msl, list(nss)[:msl], mwlt, mwlr, op_smear, tuple(alpha_action), alpha_ape,
                      tuple(alpha_hyp), proj_iter)


def wl_idx(p: WloopParms, sl1: int, sl2: int, t: int, r: int, x0: int) -> int:
    """wl_idx (wloop_parms.c:431-434)."""
    return sl1 + p.msl * (sl2 + p.msl * (t + p.mwlt * (r + p.mwlr * x0)))


def wl_array(p: WloopParms, wl_mat: np.ndarray, n0: int) -> np.ndarray:
    """wl_mat as an array indexed [x0, r, t, sl2, sl1]."""
    return wl_mat.reshape(n0, p.mwlr, p.mwlt, p.msl, p.msl)


def volume(n) -> int:
    return int(n[0]) * int(n[1]) * int(n[2]) * int(n[3])


def generate_links(n, bc: int, seed: int, eps: float) -> np.ndarray:
    """Synthetic field on the host (same bytes as Context.generate)."""
    u = np.empty((volume(n), 4, 3, 3), dtype=np.complex128)
    nn = np.asarray(n, dtype=np.int32)
    check(lib.wlg_generate_links(iptr(nn), bc, seed, eps, dptr(u.view(np.float64))),
          "generate_links")
    return u


def aux_uniform(seed: int, index: int, tag: int) -> float:
    return lib.wlg_aux_uniform(seed, index, tag)


def device_count() -> int:
    return lib.wlg_device_count()


class Context:
    """One lattice resident on one GPU (wlg_ctx)."""

    def __init__(self, n, bc: int = 3, precision: str = "fp64", device: int = 0):
        self.n = tuple(int(x) for x in n)
        self.bc = bc
        self.precision = precision
        self.vol = volume(self.n)
        nn = np.asarray(self.n, dtype=np.int32)
        h = C.c_void_p()
        check(lib.wlg_create(iptr(nn), bc, PRECISIONS[precision], device, C.byref(h)), "create")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.wlg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- fields --------------------------------------------------------------
    def upload(self, u: np.ndarray) -> None:
        u = np.ascontiguousarray(u, dtype=np.complex128)
        assert u.size == self.vol * 36
        check(lib.wlg_upload_links(self._h, dptr(u.view(np.float64))), "upload")

    def prefetch(self, u: np.ndarray) -> None:
        """Starts copying the next field to the device while the current
        measurement runs; `upload_prefetched` makes it the gauge field.  u
        must stay alive and unchanged until then (pinned memory for overlap)."""
        assert u.flags.c_contiguous and u.dtype == np.complex128 and u.size == self.vol * 36
        self._prefetch_ref = u
        check(lib.wlg_prefetch_links(self._h, dptr(u.view(np.float64))), "prefetch")

    def upload_prefetched(self) -> None:
        check(lib.wlg_upload_prefetched(self._h), "upload_prefetched")
        self._prefetch_ref = None

    def download(self) -> np.ndarray:
        u = np.empty((self.vol, 4, 3, 3), dtype=np.complex128)
        check(lib.wlg_download_links(self._h, dptr(u.view(np.float64))), "download")
        return u

    def upload_openqcd(self, ud: np.ndarray, ipt: np.ndarray) -> None:
        ud = np.ascontiguousarray(ud, dtype=np.complex128)
        ipt = np.ascontiguousarray(ipt, dtype=np.int32)
        check(lib.wlg_upload_openqcd(self._h, dptr(ud.view(np.float64)), iptr(ipt)), "upload_openqcd")

    def download_openqcd(self, ipt: np.ndarray) -> np.ndarray:
        ud = np.empty((self.vol * 4, 3, 3), dtype=np.complex128)
        ipt = np.ascontiguousarray(ipt, dtype=np.int32)
        check(lib.wlg_download_openqcd(self._h, dptr(ud.view(np.float64)), iptr(ipt)),
              "download_openqcd")
        return ud

    def generate(self, seed: int, eps: float) -> None:
        check(lib.wlg_generate(self._h, seed, eps), "generate")

    def sync(self):
        check(lib.wlg_sync(self._h), "sync")

    def free_scratch(self):
        check(lib.wlg_free_scratch(self._h), "free_scratch")

    # -- smearing (include/smear.h) -----------------------------------------
    def hyp_links(self, a1, a2, a3, proj=1, piter=4, keep=0):
        check(lib.wlg_hyp(self._h, a1, a2, a3, proj, piter, 0, 4, keep), "hyp_links")

    def hyp_time_links(self, a1, a2, a3, proj=1, piter=4, keep=0):
        check(lib.wlg_hyp(self._h, a1, a2, a3, proj, piter, 0, 1, keep), "hyp_time_links")

    def hyp_space_links(self, a1, a2, a3, proj=1, piter=4, keep=0):
        check(lib.wlg_hyp(self._h, a1, a2, a3, proj, piter, 1, 4, keep), "hyp_space_links")

    def ape_links(self, alpha, proj=1, piter=4, nsweeps=1, keep=0):
        check(lib.wlg_ape(self._h, alpha, proj, piter, 1, nsweeps, keep), "ape_links")

    def ape_spatial_links(self, alpha, proj=1, piter=4, nsweeps=1, keep=0):
        check(lib.wlg_ape(self._h, alpha, proj, piter, 0, nsweeps, keep), "ape_spatial_links")

    def hyp_spatial_links(self, a1, a2, proj=1, piter=4, nsweeps=1, keep=0):
        check(lib.wlg_hyp_spatial(self._h, a1, a2, proj, piter, nsweeps, keep), "hyp_spatial_links")

    # -- configurations in openQCD's exported format ---------------------------
    def import_cnfg(self, path: str) -> float:
        """ms10's import_cnfg (main/ms10.c:709-718) into this context: the
        field of an exported file, with its stored average plaquette checked
        against the FP64 plaquette of the links read; returns that value."""
        out = np.zeros(1)
        check(lib.wlg_import_cnfg(self._h, os.fsencode(path), dptr(out)), "import_cnfg")
        return float(out[0])

    def export_cnfg(self, path: str) -> float:
        """Writes the context's field in the exported format with its average
        plaquette in the head; returns that value."""
        out = np.zeros(1)
        check(lib.wlg_export_cnfg(self._h, os.fsencode(path), dptr(out)), "export_cnfg")
        return float(out[0])

    def average_plaquette(self) -> float:
        """lnk_plaq_sum over the number of plaquettes: 6 V, or (6 N0 - 3)
        N1 N2 N3 with open boundary conditions."""
        return self.lnk_plaq_sum() / plaquette_count(self.n, self.bc)

    # -- lnk -------------------------------------------------------------------
    def lnk_plaq_sum(self) -> float:
        out = np.zeros(1)
        check(lib.wlg_plaq_sum(self._h, dptr(out)), "lnk_plaq_sum")
        return float(out[0])

    # -- wloop (include/wloop.h) ---------------------------------------------
    def wloop_sum(self, p: WloopParms, plaq: bool = False):
        wl = np.empty(p.wls(self.n[0]))
        pl = np.zeros(WLG_MAX_SM_LEVELS)
        cp = p.to_c()
        check(lib.wlg_wloop_sum(self._h, C.byref(cp), dptr(wl), dptr(pl) if plaq else None),
              "wloop_sum")
        return (wl, pl[:p.msl]) if plaq else wl

    def measure(self, p: WloopParms, plaq: bool = False):
        """hyp_links(alpha_action) + wloop_sum, as ms10 set_data (main/ms10.c:633-646)."""
        wl = np.empty(p.wls(self.n[0]))
        pl = np.zeros(WLG_MAX_SM_LEVELS)
        cp = p.to_c()
        check(lib.wlg_measure(self._h, C.byref(cp), dptr(wl), dptr(pl) if plaq else None),
              "measure")
        return (wl, pl[:p.msl]) if plaq else wl

    def level(self, sl: int) -> np.ndarray:
        out = np.empty((self.vol, 3, 3, 3), dtype=np.complex128)
        check(lib.wlg_download_level(self._h, sl, dptr(out.view(np.float64))), "level")
        return out

    def lines(self, sl: int):
        """Spatial lines of level sl left by the last measurement: (lines of
        shape (V, 3, 3, 3), their length R = mwlr); get_pus slots msl+sl."""
        out = np.empty((self.vol, 3, 3, 3), dtype=np.complex128)
        length = C.c_int(0)
        check(lib.wlg_download_lines(self._h, sl, dptr(out.view(np.float64)), C.byref(length)),
              "lines")
        return out, length.value

    # -- timing ---------------------------------------------------------------
    def set_profiling(self, on: bool):
        check(lib.wlg_set_profiling(self._h, int(on)), "set_profiling")

    def kernel_time(self, name: str):
        ms = C.c_double()
        n = C.c_longlong()
        check(lib.wlg_kernel_time(self._h, name.encode(), C.byref(ms), C.byref(n)), "kernel_time")
        return ms.value, n.value

    def reset_kernel_times(self):
        check(lib.wlg_reset_kernel_times(self._h), "reset_kernel_times")

    def set_contract_shape(self, G=0, nCB=0, block=0):
        check(lib.wlg_set_contract_shape(self._h, G, nCB, block), "set_contract_shape")

    def set_contract_tuning(self, variant=0, G=0, SB=0, nCB=0, block=0):
        check(lib.wlg_set_contract_tuning(self._h, variant, G, SB, nCB, block),
              "set_contract_tuning")

    def set_gram_tuning(self, occ=0, ord=0, bx=0, stages=0, cpc=0):
        """Shape of the temporal-gauge form's Gram kernel (0: automatic)."""
        check(lib.wlg_set_gram_tuning(self._h, occ, ord, bx, stages, cpc), "set_gram_tuning")

    def gram_shape(self, msl: int, mwlt: int) -> dict:
        """The Gram kernel's plan for msl levels and mwlt on this lattice."""
        v = (C.c_int * 10)()
        check(lib.wlg_gram_shape(self._h, msl, mwlt, v), "gram_shape")
        keys = ("tq", "occ", "ord", "bx", "nblk", "stages", "cpc", "nsplit", "block", "smem_kib")
        return dict(zip(keys, list(v)))

    @property
    def contract_form(self) -> int:
        """Contraction form of the last measurement (11: temporal gauge; 0: none yet)."""
        f = C.c_int(0)
        check(lib.wlg_contract_form(self._h, C.byref(f)), "contract_form")
        return f.value

    @property
    def stream(self) -> int:
        """cudaStream_t of the context (for event timing by the caller)."""
        return lib.wlg_stream(self._h) or 0

    def gauge_transform(self, seed: int, eps: float = 1.0):
        """U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag with a synthetic SU(3) field g
        (openQCD's random_g + transform_ud, devel/wloop/check2.c)."""
        check(lib.wlg_gauge_transform(self._h, seed, eps), "gauge_transform")

    def shift_ud(self, s):
        """U(x) <- U(x - s) (openQCD's shift_ud, devel/wloop/check3.c)."""
        check(lib.wlg_shift_links(self._h, (C.c_int * 4)(*s)), "shift_ud")

    def snapshot(self):
        check(lib.wlg_snapshot(self._h), "snapshot")

    def restore(self):
        check(lib.wlg_restore(self._h), "restore")


def plaquette_count(n, bc: int) -> float:
    """Plaquettes lnk_plaq_sum runs over: 6 V, or (6 N0 - 3) N1 N2 N3 with open
    boundary conditions (the time plaquettes of the last slice are absent,
    lnkplaq.c:88)."""
    vs = float(n[1] * n[2] * n[3])
    return (6.0 * n[0] - 3.0 if bc == 0 else 6.0 * n[0]) * vs


def launch_count() -> int:
    return lib.wlg_launch_count()


def peak_tflops(precision: str = "mixed", device: int = 0) -> float:
    """Measured vector FMA peak: "fp64", "mixed" (scalar FP32 FMAs) or
    "f32x2" (packed two-lane FP32 FMAs)."""
    out = np.zeros(1)
    code = 2 if precision == "f32x2" else PRECISIONS[precision]
    check(lib.wlg_peak_flops(code, device, dptr(out)), "peak_flops")
    return float(out[0])


def staple_sum(n, u1: np.ndarray, u2: np.ndarray, mu: int, nu: int, vb: np.ndarray) -> None:
    """staple_sum (staple_sum.c:53-87) on AoS host fields; vb is updated."""
    nn = np.asarray(n, dtype=np.int32)
    u1 = np.ascontiguousarray(u1, dtype=np.complex128)
    u2 = np.ascontiguousarray(u2, dtype=np.complex128)
    assert vb.flags.c_contiguous and vb.dtype == np.complex128
    check(lib.wlg_staple_sum(iptr(nn), dptr(u1.view(np.float64)), dptr(u2.view(np.float64)), mu, nu,
                             dptr(vb.view(np.float64))), "staple_sum")


def approx_project_to_su3(m: np.ndarray, iterations: int) -> None:
    """approx_project_to_su3_dble (projection.c:120-154) in place on (..., 3, 3)."""
    assert m.flags.c_contiguous and m.dtype == np.complex128
    check(lib.wlg_project(dptr(m.view(np.float64)), m.size // 9, iterations), "project")


class Batch:
    """Many configurations measured together (wlg_batch): every stage is one
    kernel over all lattices and the pipeline replays as one CUDA graph."""

    def __init__(self, items, precision: str = "mixed", device: int = 0):
        """items: sequence of (n, bc, WloopParms)."""
        self.items = [(tuple(int(x) for x in n), int(bc), p) for n, bc, p in items]
        k = len(self.items)
        dims = np.asarray([n for n, _, _ in self.items], dtype=np.int32).reshape(-1)
        bcs = np.asarray([bc for _, bc, _ in self.items], dtype=np.int32)
        parr = (WlgParms * k)(*[p.to_c() for _, _, p in self.items])
        h = C.c_void_p()
        check(lib.wlg_batch_create(k, iptr(dims), iptr(bcs), parr, PRECISIONS[precision], device,
                                   C.byref(h)), "batch_create")
        self._h = h
        self.precision = precision

    def close(self):
        if getattr(self, "_h", None):
            lib.wlg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return len(self.items)

    @property
    def device_bytes(self) -> int:
        return lib.wlg_batch_bytes(self._h)

    def upload(self, i: int, u: np.ndarray):
        u = np.ascontiguousarray(u, dtype=np.complex128)
        check(lib.wlg_batch_upload(self._h, i, dptr(u.view(np.float64))), "batch_upload")

    def generate(self, seeds, eps):
        s = (C.c_uint64 * len(self.items))(*[int(x) for x in seeds])
        e = np.ascontiguousarray(eps, dtype=np.float64)
        check(lib.wlg_batch_generate(self._h, s, dptr(e)), "batch_generate")

    def snapshot(self):
        check(lib.wlg_batch_snapshot(self._h), "batch_snapshot")

    def restore(self):
        check(lib.wlg_batch_restore(self._h), "batch_restore")

    def run(self):
        check(lib.wlg_batch_run(self._h), "batch_run")

    def result(self, i: int) -> np.ndarray:
        n, _, p = self.items[i]
        out = np.empty(p.wls(n[0]))
        check(lib.wlg_batch_result(self._h, i, dptr(out)), "batch_result")
        return out

    def stats(self):
        ms = C.c_double()
        k = C.c_int()
        check(lib.wlg_batch_stats(self._h, C.byref(ms), C.byref(k)), "batch_stats")
        return ms.value, k.value

    @property
    def stream(self) -> int:
        return lib.wlg_batch_stream(self._h) or 0

    def set_contract_shape(self, G=0, SB=0, nCB=0, block=0):
        check(lib.wlg_batch_set_contract_shape(self._h, G, SB, nCB, block),
              "batch_set_contract_shape")


def estimate_bytes(n, bc: int, p: WloopParms, precision: str = "mixed") -> int:
    """Device bytes one measurement of this lattice holds in a batch."""
    nn = np.asarray(n, dtype=np.int32)
    b = np.asarray([bc], dtype=np.int32)
    cp = p.to_c()
    return int(lib.wlg_batch_estimate_bytes(1, iptr(nn), iptr(b), C.byref(cp), PRECISIONS[precision]))


class Server:
    """Measurement request loop with continuous batching (wlg_server)."""

    def __init__(self, device: int = 0, mem_fraction: float = 0.8, max_inflight: int = 2,
                 max_batch: int = 8):
        h = C.c_void_p()
        if lib.wlg_server_create(device, mem_fraction, max_inflight, max_batch, C.byref(h)) != 0:
            raise WlgError("server_create failed (no device or bad arguments)")
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib.wlg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def budget(self) -> int:
        return int(lib.wlg_server_budget(self._h))

    def set_limits(self, budget_bytes: int = 0, bypass_ms: float = -1.0) -> None:
        """Memory budget in bytes (> 0 replaces it) and the time the head of
        the queue may be bypassed by later requests that fit (>= 0)."""
        check(lib.wlg_server_set_limits(self._h, int(budget_bytes), float(bypass_ms)),
              "server_set_limits")

    def submit(self, n, bc: int, p: WloopParms, precision: str = "mixed", seed: int = 0,
               eps: float = 0.2, links: Optional[np.ndarray] = None) -> int:
        r = WlgRequest()
        for i in range(4):
            r.n[i] = int(n[i])
        r.bc = bc
        r.parms = p.to_c()
        r.precision = PRECISIONS[precision]
        r.seed = int(seed)
        r.eps = float(eps)
        if links is not None:
            links = np.ascontiguousarray(links, dtype=np.complex128)
            r.links = dptr(links.view(np.float64))
        rid = lib.wlg_server_submit(self._h, C.byref(r))
        if rid < 0:
            raise WlgError("server_submit: bad request")
        self._nwl = getattr(self, "_nwl", {})
        self._nwl[rid] = p.wls(int(n[0]))
        return rid

    def wait(self, rid: int):
        out = np.empty(self._nwl[rid])
        lat = C.c_double()
        bs = C.c_int()
        if lib.wlg_server_wait(self._h, rid, dptr(out), C.byref(lat), C.byref(bs)) != 0:
            raise WlgError("request %d failed: %s" % (rid, lib.wlg_server_error().decode()))
        lib.wlg_server_release(self._h, rid)
        return out, lat.value, bs.value

    def stats(self) -> dict:
        c, f, b = C.c_longlong(), C.c_longlong(), C.c_longlong()
        p50, p99, thr = C.c_double(), C.c_double(), C.c_double()
        check(lib.wlg_server_stats(self._h, C.byref(c), C.byref(f), C.byref(b), C.byref(p50),
                                   C.byref(p99), C.byref(thr)), "server_stats")
        return {"completed": c.value, "failed": f.value, "batches": b.value,
                "p50_ms": p50.value, "p99_ms": p99.value, "throughput": thr.value}
