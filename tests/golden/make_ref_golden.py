"""Golden fixtures from the reference itself (oracle/_ref, built by
`make -C oracle ref`): the reference's own modules run ms10's
per-configuration work (hyp_links, then wloop_sum; main/ms10.c:633-646) on
the synthetic fields of the benchmark configurations, and the Wilson loops
on the time slices that the oracle's fixtures store are written next to them:

  ref_c2_24x24x24x48_open.npz        c2 (24^3x48, open bc, msl 5, r<=12, t<=16)
  ref_c4_00_16x16x16x32_periodic.npz configuration 0 of the 64-configuration batch
  ref_c4_48_24x24x24x48_periodic.npz configuration 48 of the batch

The reference runs on one core (no MPI): c2 takes about 20 minutes, c4_48
about 10, c4_00 about one.  The inputs come from the oracle's copy of the
generator (oracle/fieldgen.c), the same bytes as the product's, and each file
records their sha256.  Run: python tests/golden/make_ref_golden.py [name ...]
(each configuration in its own process, since one reference library holds
one lattice).
"""
import hashlib
import multiprocessing as mp
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

NAMES = ["c2_24x24x24x48_open", "c4_00_16x16x16x32_periodic", "c4_48_24x24x24x48_periodic"]


def run(name):
    from tests import oracle as O
    from tests import refimpl as R
    from wloop_b200.api import WloopParms
    f = dict(np.load(os.path.join(HERE, name + ".npz")))
    n = tuple(int(x) for x in f["n"])
    bc = int(f["bc"])
    p = WloopParms(msl=int(f["msl"]), nss=[int(x) for x in f["nss"]], mwlt=int(f["mwlt"]),
                   mwlr=int(f["mwlr"]), alpha_ape=float(f["alpha_ape"]),
                   alpha_action=tuple(f["alpha_action"]), proj_iter=int(f["proj_iter"]))
    O.set_threads(1)
    u = O.generate_links(n, bc, int(f["seed"]), float(f["eps"]))
    sha = hashlib.sha256(u.view(np.uint8)).hexdigest()
    assert sha == str(f["sha256"]), "input differs from the oracle fixture's"
    ref = R.Ref(n)
    ref.set_field(bc, u)
    wl = ref.measure(p).reshape(n[0], -1)
    np.savez_compressed(os.path.join(HERE, "ref_" + name + ".npz"), sha256=sha, x0=f["x0"],
                        wl=wl[f["x0"]], plaq_hyp=ref.plaq_sum())
    return name


if __name__ == "__main__":
    todo = sys.argv[1:] or NAMES
    with mp.get_context("spawn").Pool(len(todo)) as pool:
        for name in pool.imap_unordered(run, todo):
            print("wrote ref_" + name + ".npz", flush=True)
