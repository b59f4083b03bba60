"""ctypes binding of libwloop_b200.so (the C ABI in include/wloop_b200.h).

The library is built in-tree by ``python wloop_b200/build.py``.  Importing
this module without the built library raises: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libwloop_b200.so")

WLG_MAX_SM_LEVELS = 8
WLG_FP64 = 0
WLG_MIXED = 1
WLG_OP_APE = 0
WLG_OP_HYP = 1


class WlgParms(C.Structure):
    """Mirror of wlg_wloop_parms (include/wloop_b200.h)."""
    _fields_ = [
        ("msl", C.c_int),
        ("nss", C.c_int * WLG_MAX_SM_LEVELS),
        ("mwlt", C.c_int),
        ("mwlr", C.c_int),
        ("op_smear", C.c_int),
        ("alpha_action", C.c_double * 3),
        ("alpha_ape", C.c_double),
        ("alpha_hyp", C.c_double * 2),
        ("proj_iter", C.c_int),
    ]


class WlgRequest(C.Structure):
    """Mirror of wlg_request (include/wloop_b200.h)."""
    _fields_ = [
        ("n", C.c_int * 4),
        ("bc", C.c_int),
        ("parms", WlgParms),
        ("precision", C.c_int),
        ("seed", C.c_uint64),
        ("eps", C.c_double),
        ("links", C.POINTER(C.c_double)),
    ]


class WlgError(RuntimeError):
    pass


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"wloop_b200: native library {LIB_PATH} is not built; run "
            "`python wloop_b200/build.py` (the CUDA path has no CPU fallback)")
    lib = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
    vp, ip, dp, i, d = C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.c_int, C.c_double
    u64, u32 = C.c_uint64, C.c_uint32
    sig = {
        "wlg_last_error": (C.c_char_p, []),
        "wlg_device_count": (i, []),
        "wlg_version": (i, []),
        "wlg_create": (i, [ip, i, i, i, C.POINTER(vp)]),
        "wlg_destroy": (i, [vp]),
        "wlg_sync": (i, [vp]),
        "wlg_free_scratch": (i, [vp]),
        "wlg_upload_links": (i, [vp, dp]),
        "wlg_download_links": (i, [vp, dp]),
        "wlg_prefetch_links": (i, [vp, dp]),
        "wlg_upload_prefetched": (i, [vp]),
        "wlg_upload_openqcd": (i, [vp, dp, ip]),
        "wlg_download_openqcd": (i, [vp, dp, ip]),
        "wlg_generate": (i, [vp, u64, d]),
        "wlg_generate_links": (i, [ip, i, u64, d, dp]),
        "wlg_aux_uniform": (d, [u64, u64, u32]),
        "wlg_hyp": (i, [vp, d, d, d, i, i, i, i, i]),
        "wlg_ape": (i, [vp, d, i, i, i, i, i]),
        "wlg_hyp_spatial": (i, [vp, d, d, i, i, i, i]),
        "wlg_plaq_sum": (i, [vp, dp]),
        "wlg_wloop_sum": (i, [vp, C.POINTER(WlgParms), dp, dp]),
        "wlg_measure": (i, [vp, C.POINTER(WlgParms), dp, dp]),
        "wlg_download_level": (i, [vp, i, dp]),
        "wlg_download_lines": (i, [vp, i, dp, ip]),
        "wlg_staple_sum": (i, [ip, dp, dp, i, i, dp]),
        "wlg_project": (i, [dp, i, i]),
        "wlg_set_profiling": (i, [vp, i]),
        "wlg_kernel_time": (i, [vp, C.c_char_p, dp, C.POINTER(C.c_longlong)]),
        "wlg_reset_kernel_times": (i, [vp]),
        "wlg_set_contract_shape": (i, [vp, i, i, i]),
        "wlg_set_contract_tuning": (i, [vp, i, i, i, i, i]),
        "wlg_stream": (vp, [vp]),
        "wlg_contract_form": (i, [vp, ip]),
        "wlg_set_gram_tuning": (i, [vp, i, i, i, i, i]),
        "wlg_gram_shape": (i, [vp, i, i, ip]),
        "wlg_gram_plan_shape": (i, [ip, i, i, i, i, ip, C.POINTER(C.c_longlong)]),
        "wlg_launch_count": (C.c_longlong, []),
        "wlg_snapshot": (i, [vp]),
        "wlg_gauge_transform": (i, [vp, u64, d]),
        "wlg_shift_links": (i, [vp, ip]),
        "wlg_restore": (i, [vp]),
        "wlg_peak_flops": (i, [i, i, dp]),
        "wlg_selftest_wait": (i, [i, d, ip, dp]),
        "wlg_batch_create": (i, [i, ip, ip, C.POINTER(WlgParms), i, i, C.POINTER(vp)]),
        "wlg_batch_destroy": (i, [vp]),
        "wlg_batch_size": (i, [vp]),
        "wlg_batch_bytes": (C.c_longlong, [vp]),
        "wlg_batch_upload": (i, [vp, i, dp]),
        "wlg_batch_generate": (i, [vp, C.POINTER(u64), dp]),
        "wlg_batch_snapshot": (i, [vp]),
        "wlg_batch_restore": (i, [vp]),
        "wlg_batch_run": (i, [vp]),
        "wlg_batch_result": (i, [vp, i, dp]),
        "wlg_batch_stats": (i, [vp, dp, ip]),
        "wlg_batch_stream": (vp, [vp]),
        "wlg_batch_set_contract_shape": (i, [vp, i, i, i, i]),
        "wlg_plaq_sum_noalloc": (i, [vp, ip, i, vp, vp]),
        "wlg_batch_use_graph": (i, [vp, i]),
        "wlg_batch_pool_idle_bytes": (C.c_longlong, [i]),
        "wlg_batch_estimate_bytes": (C.c_longlong, [i, ip, ip, C.POINTER(WlgParms), i]),
        "wlg_server_create": (i, [i, d, i, i, C.POINTER(vp)]),
        "wlg_server_destroy": (i, [vp]),
        "wlg_server_submit": (C.c_longlong, [vp, C.POINTER(WlgRequest)]),
        "wlg_server_wait": (i, [vp, C.c_longlong, dp, dp, ip]),
        "wlg_server_release": (i, [vp, C.c_longlong]),
        "wlg_server_error": (C.c_char_p, []),
        "wlg_server_stats": (i, [vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                 C.POINTER(C.c_longlong), dp, dp, dp]),
        "wlg_server_budget": (C.c_longlong, [vp]),
        "wlg_server_set_limits": (i, [vp, C.c_longlong, d]),
        "wlg_dat_error": (C.c_char_p, []),
        "wlg_dat_head": (i, [C.POINTER(WlgParms), i, ip]),
        "wlg_dat_write_head": (i, [C.c_char_p, ip]),
        "wlg_dat_check_head": (i, [C.c_char_p, ip]),
        "wlg_dat_append": (i, [C.c_char_p, i, dp, i]),
        "wlg_dat_count": (C.c_longlong, [C.c_char_p, ip]),
        "wlg_dat_read": (i, [C.c_char_p, C.c_longlong, ip, dp, i]),
        "wlg_par_write_wloop": (i, [C.c_char_p, C.POINTER(WlgParms)]),
        "wlg_par_check_wloop": (i, [C.c_char_p, C.c_longlong, C.POINTER(WlgParms)]),
        "wlg_cnfg_error": (C.c_char_p, []),
        "wlg_cnfg_read_head": (i, [C.c_char_p, ip, dp]),
        "wlg_cnfg_import": (i, [C.c_char_p, ip, dp, dp]),
        "wlg_cnfg_export": (i, [C.c_char_p, ip, dp, d]),
        "wlg_import_cnfg": (i, [vp, C.c_char_p, dp]),
        "wlg_export_cnfg": (i, [vp, C.c_char_p, dp]),
        "wlg_par_write_bc": (i, [C.c_char_p, i]),
        "wlg_par_check_bc": (i, [C.c_char_p, C.c_longlong, i]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


lib = _load()


def check(rc: int, what: str = "") -> None:
    if rc != 0:
        msg = lib.wlg_last_error().decode(errors="replace")
        raise WlgError(f"{what}: {msg}" if what else msg)


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))
