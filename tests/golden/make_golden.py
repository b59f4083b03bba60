"""Generates the golden fixtures in tests/golden/ from the FP64 oracle.

The reference ships no golden vectors and cannot be built here, so these
fixtures freeze the oracle's output (itself pinned by the reference's
property checks in tests/test_oracle.py) on the synthetic fields of the
benchmark configurations, for the GPU parity tests at full size:

  c1_8x8x8x8_periodic.npz   full wl_mat and |terms| sums (2048 entries)
  c2_24x24x24x48_open.npz   wl_mat and |terms| sums on time slices 0 and 40
                            (4800 entries each) and the per-level plaquettes
  c3_32x32x32x64_periodic.npz  the same on time slices 0 and 37 (13824
                            entries each) of the 32^3x64 bench workload
  c4_00_16x16x16x32_periodic.npz  configuration 0 of the 64-configuration
                            batch (16^3x32, its own seed and eps), 8 time
                            slices of 1296 entries
  c4_48_24x24x24x48_periodic.npz  configuration 48 of the batch (the first
                            24^3x48), 8 time slices of 2704 entries

Each file records the sha256 of the generated input field so a test can
prove it regenerated the same bytes.  Run: python tests/golden/make_golden.py [c1] [c2] [c3]
(c2 takes about ten minutes on 8 cores, c3 about 45 minutes, c4 about
three minutes).
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from tests import oracle as O  # noqa: E402
from wloop_b200.api import generate_links  # noqa: E402
from wloop_b200.workloads import C1, C2, C3, batch_workloads  # noqa: E402


def field_sha(u):
    return hashlib.sha256(np.ascontiguousarray(u).view(np.uint8)).hexdigest()


def run(w, slices=None):
    p = w.parms
    u = generate_links(w.n, w.bc, w.seed, w.eps)
    sha = field_sha(u)
    uh = O.hyp_links(w.n, w.bc, u, *p.alpha_action, p.proj, p.proj_iter)
    plaq_hyp = O.plaq_sum(w.n, w.bc, uh)
    wl, wa, pl = O.wloop_sum(w.n, w.bc, uh, p, want_abs=True, want_plaq=True)
    n0 = w.n[0]
    wl = wl.reshape(n0, -1)
    wa = wa.reshape(n0, -1)
    out = dict(n=np.array(w.n), bc=w.bc, seed=w.seed, eps=w.eps, sha256=sha,
               msl=p.msl, nss=np.array(p.nss), mwlt=p.mwlt, mwlr=p.mwlr,
               alpha_ape=p.alpha_ape, proj_iter=p.proj_iter,
               alpha_action=np.array(p.alpha_action), plaq_hyp=plaq_hyp, plaq_levels=pl)
    if slices is None:
        out.update(x0=np.arange(n0), wl=wl, wl_abs=wa)
    else:
        out.update(x0=np.array(slices), wl=wl[slices], wl_abs=wa[slices])
    return out


def main(which):
    O.set_threads(os.cpu_count() or 1)
    if "c1" in which:
        np.savez_compressed(os.path.join(HERE, "c1_8x8x8x8_periodic.npz"), **run(C1))
    if "c2" in which:
        np.savez_compressed(os.path.join(HERE, "c2_24x24x24x48_open.npz"), **run(C2, [0, 40]))
    if "c3" in which:
        np.savez_compressed(os.path.join(HERE, "c3_32x32x32x64_periodic.npz"), **run(C3, [0, 37]))
    if "c4" in which:
        ws = batch_workloads()
        for i in (0, 48):
            w = ws[i]
            n0, ns = w.n[0], w.n[1]
            slices = sorted({(k * n0) // 8 + (k % 3) for k in range(8)})
            name = f"c4_{i:02d}_{ns}x{ns}x{ns}x{n0}_periodic.npz"
            np.savez_compressed(os.path.join(HERE, name), batch_index=i, **run(w, slices))


if __name__ == "__main__":
    main(sys.argv[1:] or ["c1", "c2"])
