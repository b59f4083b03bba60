"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the
oracle) at the full sizes of the 8^4, 24^3x48 and 32^3x64 configurations
(the last is the bench workload: HYP2, 50 APE sweeps over 6 levels, all
loops r <= 16, t <= 24; two of its 64 time slices are stored).

CPU: the synthetic input is regenerated bit for bit (sha256 of the field),
and the oracle reproduces the c1 fixture.  GPU: the FP64 path matches every
stored entry to 1e-12 (scaled by max(|W|, sum|terms|/norm)) and the
per-level plaquettes to 1e-12; the mixed path stays within 1e-6.
"""
import hashlib
import os

import numpy as np
import pytest

from tests import oracle as O
from wloop_b200.api import WloopParms, generate_links
from wloop_b200.workloads import C1, C2, C3

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(HERE, name)))


def parms(f):
    return WloopParms(msl=int(f["msl"]), nss=[int(x) for x in f["nss"]], mwlt=int(f["mwlt"]),
                      mwlr=int(f["mwlr"]), alpha_ape=float(f["alpha_ape"]),
                      alpha_action=tuple(f["alpha_action"]), proj_iter=int(f["proj_iter"]))


def field(f):
    n = tuple(int(x) for x in f["n"])
    return n, int(f["bc"]), generate_links(n, int(f["bc"]), int(f["seed"]), float(f["eps"]))


ALL = ["c1_8x8x8x8_periodic.npz", "c2_24x24x24x48_open.npz", "c3_32x32x32x64_periodic.npz"]


@pytest.mark.parametrize("name", ALL)
def test_fixture_input_regenerates(name):
    f = load(name)
    _, _, u = field(f)
    assert hashlib.sha256(u.view(np.uint8)).hexdigest() == str(f["sha256"])


def test_fixture_matches_workload_definitions():
    for name, w in zip(ALL, (C1, C2, C3)):
        f = load(name)
        assert tuple(f["n"]) == w.n and int(f["bc"]) == w.bc and int(f["seed"]) == w.seed
        assert int(f["msl"]) == w.parms.msl and list(f["nss"]) == list(w.parms.nss)


def test_oracle_reproduces_c1():
    f = load("c1_8x8x8x8_periodic.npz")
    n, bc, u = field(f)
    p = parms(f)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    wl = O.wloop_sum(n, bc, uh, p).reshape(n[0], -1)
    scale = np.maximum(np.abs(f["wl"]), f["wl_abs"])
    assert (np.abs(wl - f["wl"]) / scale).max() < 1e-13


def _check(got, f, tol):
    ref, ref_abs = f["wl"], f["wl_abs"]
    zero = ref == 0.0
    assert np.all(got[zero] == 0.0)
    err = np.abs(got - ref)[~zero] / np.maximum(np.abs(ref), ref_abs)[~zero]
    return err.max()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ALL)
def test_gpu_fp64_matches_fixture(name):
    from wloop_b200 import Context
    f = load(name)
    n, bc, u = field(f)
    p = parms(f)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        wl, plaq = c.measure(p, plaq=True)
    got = wl.reshape(n[0], -1)[f["x0"]]
    assert _check(got, f, 1e-12) <= 1e-12
    assert np.abs(plaq - f["plaq_levels"]).max() / np.abs(f["plaq_levels"]).max() < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", ALL)
def test_gpu_mixed_within_1e6_of_fixture(name):
    from wloop_b200 import Context
    f = load(name)
    n, bc, u = field(f)
    p = parms(f)
    with Context(n, bc, "mixed") as c:
        c.upload(u)
        wl = c.measure(p)
    got = wl.reshape(n[0], -1)[f["x0"]]
    err = _check(got, f, 1e-6)
    print(f"{name}: mixed max scaled error {err:.2e}")
    assert err <= 1e-6
    if name.startswith("c3"):
        # the headline workload: every stored W within 1e-6 relative of the
        # FP64 oracle, without the |terms| scale
        nz = f["wl"] != 0.0
        rel = np.abs(got - f["wl"])[nz] / np.abs(f["wl"])[nz]
        print(f"{name}: mixed max relative error {rel.max():.2e}")
        assert rel.max() <= 1e-6
