"""wloop_b200 -- B200 (sm_100a) implementation of the wloop measurement path.

HYP smearing of the gauge links, APE / spatial-HYP smearing of the spatial
links over several levels, temporal and spatial line products and the
time-slice resolved Wilson-loop correlation matrices W(sl1,sl2;t,r;x0),
behind the C ABI of include/wloop_b200.h.  Importing the package loads the
native library and fails if it is not built.
"""
from ._native import WlgError, lib  # noqa: F401  (raises ImportError if unbuilt)
from .api import (APE, HYP, Context, WloopParms, aux_uniform, approx_project_to_su3,  # noqa: F401
                  device_count, generate_links, set_wloop_parms, staple_sum, wl_array, wl_idx)

__all__ = ["APE", "HYP", "Context", "WloopParms", "WlgError", "aux_uniform",
           "approx_project_to_su3", "device_count", "generate_links", "set_wloop_parms",
           "staple_sum", "wl_array", "wl_idx"]
