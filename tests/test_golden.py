"""Golden fixtures (tests/golden/, made by tests/golden/make_golden.py from the
oracle) at the full sizes of the 8^4, 24^3x48 and 32^3x64 configurations
(the last is the bench workload: HYP2, 50 APE sweeps over 6 levels, all
loops r <= 16, t <= 24; two of its 64 time slices are stored).

CPU: the synthetic input is regenerated bit for bit (sha256 of the field),
and the oracle reproduces the c1 fixture.  GPU: the FP64 path matches every
stored entry to 1e-12 (scaled by max(|W|, sum|terms|/norm)) and the
per-level plaquettes to 1e-12; the mixed path stays within 1e-6 plain
relative on every non-zero entry.  Two configurations of the 64-configuration
batch (tests/golden/c4_*.npz) are checked inside the full batch run.
With WLG_ERROR_TABLE_DIR set, the mixed tests write the per-W(sl1,sl2;t,r)
error table there.
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
C4 = ["c4_00_16x16x16x32_periodic.npz", "c4_48_24x24x24x48_periodic.npz"]


@pytest.mark.parametrize("name", ALL + C4)
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


def _plain_rel(got, f):
    nz = f["wl"] != 0.0
    return np.abs(got - f["wl"])[nz] / np.abs(f["wl"])[nz]


def error_table(got, f, p):
    """Plain relative error of every W(sl1,sl2;t,r), max over the stored time
    slices, as an array [r][t][sl2][sl1] (the wl_idx order without x0,
    modules/wloop/wloop_parms.c:431-434); entries that are exactly zero in the
    oracle count as 0 (they are checked to be exactly zero)."""
    ref = f["wl"]
    rel = np.where(ref != 0.0, np.abs(got - ref) / np.where(ref != 0.0, np.abs(ref), 1.0), 0.0)
    return rel.reshape(len(f["x0"]), p.mwlr, p.mwlt, p.msl, p.msl).max(axis=0)


def write_error_table(path, name, tab, p):
    """One line per (t, r) with the msl x msl errors in (sl1, sl2) order."""
    with open(path, "w") as fo:
        fo.write(f"# {name}: mixed form vs the FP64 oracle, plain relative error of "
                 f"W(sl1,sl2;t,r), max over the stored time slices\n")
        fo.write("# columns: t r then sl1,sl2 = " +
                 " ".join(f"{a}{b}" for a in range(p.msl) for b in range(p.msl)) + "\n")
        for t in range(p.mwlt):
            for r in range(p.mwlr):
                vals = " ".join(f"{tab[r, t, b, a]:.1e}" for a in range(p.msl)
                                for b in range(p.msl))
                fo.write(f"{t + 1} {r + 1} {vals}\n")


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
    err = _check(got, f, 1e-12)
    rel = _plain_rel(got, f)
    print(f"{name}: fp64 max scaled error {err:.2e}, max plain relative {rel.max():.2e}, "
          f"entries above 1e-12 plain: {int(np.sum(rel > 1e-12))} of {rel.size}")
    assert err <= 1e-12
    # the full-size fixtures hold no near-zero W: every entry also within
    # 1e-12 plain relative
    assert rel.max() <= 1e-12
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
    rel = _plain_rel(got, f)
    print(f"{name}: mixed max scaled error {err:.2e}, max plain relative {rel.max():.2e}")
    out = os.environ.get("WLG_ERROR_TABLE_DIR")
    if out:
        write_error_table(os.path.join(out, "mixed_error_" + name.replace(".npz", ".txt")),
                          name, error_table(got, f, p), p)
    # every stored non-zero W within 1e-6 plain relative of the FP64 oracle
    assert rel.max() <= 1e-6



def test_c4_fixtures_are_batch_members():
    from wloop_b200.workloads import batch_workloads
    ws = batch_workloads()
    for name in C4:
        f = load(name)
        w = ws[int(f["batch_index"])]
        assert tuple(f["n"]) == w.n and int(f["seed"]) == w.seed
        assert float(f["eps"]) == w.eps and list(f["nss"]) == list(w.parms.nss)
        assert int(f["mwlt"]) == w.parms.mwlt and int(f["mwlr"]) == w.parms.mwlr


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_gpu_c4_batch_members_match_fixtures(prec):
    """The 64-configuration batch as the bench runs it (one graph launch, the
    tuner's contraction shape): configurations 0 (16^3x32) and 48 (24^3x48)
    against the oracle at their full sizes."""
    from wloop_b200.api import Batch
    from wloop_b200.autotune import tune_batch
    from wloop_b200.workloads import batch_workloads
    ws = batch_workloads()
    with Batch([(w.n, w.bc, w.parms) for w in ws], prec) as b:
        b.generate([w.seed for w in ws], [w.eps for w in ws])
        b.snapshot()
        shape = tune_batch(b)
        b.restore()
        b.run()
        for name in C4:
            f = load(name)
            i = int(f["batch_index"])
            n0 = ws[i].n[0]
            got = b.result(i).reshape(n0, -1)[f["x0"]]
            err = _check(got, f, 1e-12)
            rel = _plain_rel(got, f)
            print(f"{name} ({prec}, shape {shape}): max scaled {err:.2e}, "
                  f"max plain relative {rel.max():.2e}")
            if prec == "fp64":
                assert err <= 1e-12
            else:
                assert rel.max() <= 1e-6
            rpath = os.path.join(HERE, "ref_" + name)
            if os.path.exists(rpath):
                # the same against the reference's own output
                rf = dict(f, wl=dict(np.load(rpath))["wl"])
                if prec == "fp64":
                    assert _check(got, rf, 1e-12) <= 1e-12
                else:
                    assert _plain_rel(got, rf).max() <= 1e-6


# ---------------------------------------------------------------------------
# fixtures made by the reference itself (tests/golden/make_ref_golden.py)
# ---------------------------------------------------------------------------
REF = ["c2_24x24x24x48_open", "c4_00_16x16x16x32_periodic", "c4_48_24x24x24x48_periodic"]


def load_ref(name):
    path = os.path.join(HERE, "ref_" + name + ".npz")
    if not os.path.exists(path):
        pytest.skip(f"no reference fixture ref_{name}.npz")
    return dict(np.load(path))


@pytest.mark.parametrize("name", REF)
def test_oracle_fixture_matches_reference_fixture(name):
    """The oracle's full-size fixture against the reference's own output on
    the same field (same sha256) and time slices."""
    f, r = load(name + ".npz"), load_ref(name)
    assert str(r["sha256"]) == str(f["sha256"])
    assert np.array_equal(r["x0"], f["x0"])
    assert _check(r["wl"], f, 1e-13) <= 1e-13


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_gpu_c2_matches_reference_fixture(prec):
    from wloop_b200 import Context
    name = "c2_24x24x24x48_open"
    f, r = load(name + ".npz"), load_ref(name)
    n, bc, u = field(f)
    with Context(n, bc, prec) as c:
        c.upload(u)
        got = c.measure(parms(f)).reshape(n[0], -1)[f["x0"]]
    ref = dict(f, wl=r["wl"])  # the reference's W with the oracle's |terms| scale
    err = _check(got, ref, 1e-12)
    rel = _plain_rel(got, ref)
    print(f"{name} {prec} vs reference: max scaled {err:.2e}, max plain relative {rel.max():.2e}")
    if prec == "fp64":
        assert err <= 1e-12
    else:
        assert rel.max() <= 1e-6
