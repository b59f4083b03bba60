"""Parity pinned to the reference itself.

oracle/_ref holds the reference's own modules/{lnk,smear,wloop} compiled
unchanged from their sources against a one-process openQCD-1.4 interface
(oracle/refshim).  CPU: the oracle (the restatement every other test uses)
against the reference, function by function and for ms10's whole
per-configuration measurement.  GPU: the CUDA path through the C ABI
against the reference directly.  The two differ only in the order of the
floating-point sums over sites (openQCD numbers even sites first), so the
bars are 1e-13 (smeared links, element-wise absolute; plaquettes, relative)
and, for Wilson loops, 1e-13 (oracle) / 1e-12 (GPU FP64) of max(|W|,
sum|terms|/norm), with exact zeros exact; the mixed form stays within 1e-6
plain relative of the reference on every non-zero entry.

The reference needs even extents (its even/odd site order), so the odd
lattices of the other parity tests have no reference build.
"""
import numpy as np
import pytest

from tests import oracle as O
from tests import refimpl as R
from wloop_b200.api import APE, HYP, WloopParms

CASES = [
    ((8, 8, 8, 8), 3, WloopParms(msl=4, nss=[0, 5, 5, 5], mwlt=4, mwlr=4, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((8, 8, 8, 8), 0, WloopParms(msl=4, nss=[0, 5, 5, 5], mwlt=4, mwlr=4, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((8, 4, 6, 4), 0, WloopParms(msl=3, nss=[0, 2, 2], mwlt=5, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((8, 4, 6, 4), 3, WloopParms(msl=2, nss=[0, 3], mwlt=5, mwlr=3, op_smear=APE, alpha_ape=0.5,
                                 proj_iter=4)),
    ((6, 4, 4, 4), 3, WloopParms(msl=3, nss=[0, 1, 2], mwlt=4, mwlr=3, op_smear=HYP,
                                 alpha_hyp=(0.75, 0.3), proj_iter=4)),
    ((4, 4, 4, 4), 0, WloopParms(msl=5, nss=[0, 1, 0, 1, 1], mwlt=3, mwlr=3, op_smear=APE,
                                 alpha_ape=0.4, proj_iter=0)),
    ((10, 6, 6, 6), 0, WloopParms(msl=6, nss=[0, 2, 2, 2, 2, 2], mwlt=6, mwlr=4, op_smear=APE,
                                  alpha_ape=0.5, proj_iter=4)),
    ((6, 4, 6, 4), 0, WloopParms(msl=7, nss=[0, 1, 1, 1, 1, 1, 1], mwlt=4, mwlr=3,
                                 op_smear=APE, alpha_ape=0.5, proj_iter=4)),
    ((4, 4, 4, 6), 3, WloopParms(msl=8, nss=[1, 1, 0, 1, 1, 1, 0, 1], mwlt=3, mwlr=3,
                                 op_smear=HYP, alpha_hyp=(0.6, 0.3), proj_iter=3)),
    ((16, 8, 8, 8), 3, WloopParms(msl=3, nss=[0, 3, 3], mwlt=8, mwlr=5, op_smear=APE,
                                  alpha_ape=0.5, proj_iter=4)),
]


def need(n):
    if not R.available(n):
        pytest.skip(f"reference not built for {n} (oracle/Makefile ref)")
    return R.Ref(n)


def scaled_err(got, ref, ref_abs):
    zero = ref == 0.0
    assert np.all(got[zero] == 0.0), "exact zeros (open-bc crossing loops) must stay exact"
    return (np.abs(got - ref)[~zero] / np.maximum(np.abs(ref), ref_abs)[~zero]).max()


def test_generator_copy_matches_product():
    from wloop_b200.api import aux_uniform, generate_links
    for n, bc, seed, eps in [((8, 4, 6, 4), 0, 7, 0.3), ((4, 4, 4, 6), 3, 2 ** 40 + 3, 0.25)]:
        a = generate_links(n, bc, seed, eps)
        b = O.generate_links(n, bc, seed, eps)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
    for s, i, t in [(5000, 3, 7), (1000, 0, 1), (2 ** 33 + 1, 2 ** 35, 4)]:
        assert aux_uniform(s, i, t) == O.aux_uniform(s, i, t)


def test_field_roundtrip_through_openqcd_layout():
    n = (8, 4, 6, 4)
    ref = need(n)
    u = O.generate_links(n, 3, 11, 0.3)
    ref.set_field(3, u)
    assert np.array_equal(ref.get_field(), u)
    u0 = O.generate_links(n, 0, 11, 0.3)
    ref.set_field(0, u0)
    assert np.array_equal(ref.get_field(), u0)


def test_projection_matches_reference():
    ref = need((8, 8, 8, 8))
    rng = np.random.default_rng(1)
    m = rng.normal(size=(40, 3, 3)) + 1j * rng.normal(size=(40, 3, 3))
    m[0] = 0.0  # below the norm guard (projection.c:136)
    for it in (0, 1, 4, 10):
        a = ref.project(m, it)
        b = O.project(m, it)
        assert np.abs(a - b).max() < 1e-14


@pytest.mark.parametrize("bc", [0, 3])
@pytest.mark.parametrize("which", [0, 1, 2])
def test_hyp_matches_reference(bc, which):
    n = (8, 4, 6, 4)
    ref = need(n)
    u = O.generate_links(n, bc, 21 + which, 0.3)
    ref.set_field(bc, u)
    ref.hyp_links(1.0, 1.0, 0.5, 1, 4, which=which)
    time, space = {0: (1, 1), 1: (1, 0), 2: (0, 1)}[which]
    want = O.hyp_links(n, bc, u, 1.0, 1.0, 0.5, 1, 4, time=time, space=space)
    assert np.abs(ref.get_field() - want).max() < 1e-13


@pytest.mark.parametrize("time", [0, 1])
def test_ape_matches_reference(time):
    n = (8, 4, 6, 4)
    ref = need(n)
    u = O.generate_links(n, 3, 31, 0.3)
    ref.set_field(3, u)
    ref.ape_links(0.5, 1, 4, time=time, nsweeps=3)
    want = O.ape_links(n, u, 0.5, 1, 4, time=time, nsweeps=3)
    assert np.abs(ref.get_field() - want).max() < 1e-13


def test_hyp_spatial_matches_reference():
    n = (6, 4, 4, 4)
    ref = need(n)
    u = O.generate_links(n, 3, 41, 0.3)
    ref.set_field(3, u)
    ref.hyp_spatial_links(0.75, 0.3, 1, 4, nsweeps=2)
    want = O.hyp_spatial_links(n, u, 0.75, 0.3, 1, 4, nsweeps=2)
    assert np.abs(ref.get_field() - want).max() < 1e-13


@pytest.mark.parametrize("bc", [0, 3])
def test_plaquette_matches_reference(bc):
    n = (8, 8, 8, 8)
    ref = need(n)
    u = O.generate_links(n, bc, 51, 0.3)
    ref.set_field(bc, u)
    a, b = ref.plaq_sum(), O.plaq_sum(n, bc, u)
    assert abs(a - b) <= 1e-13 * abs(b)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_oracle_measurement_matches_reference(case):
    """ms10's per-configuration work (hyp_links, then wloop_sum) in the
    reference against the oracle on the same field."""
    n, bc, p = CASES[case]
    ref = need(n)
    u = O.generate_links(n, bc, 100 + case, 0.25)
    ref.set_field(bc, u)
    got = ref.measure(p)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    want, want_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    assert scaled_err(got, want, want_abs) <= 1e-13
    # the HYP-smeared field the reference leaves behind equals the oracle's
    assert np.abs(ref.get_field() - uh).max() < 1e-13


# 131,072 sites: above the size from which a context measures in the
# temporal gauge by default
LARGE = [((32, 16, 16, 16), bc, WloopParms(msl=3, nss=[0, 2, 2], mwlt=3, mwlr=2, op_smear=APE,
                                           alpha_ape=0.5, proj_iter=4)) for bc in (3, 0)]


@pytest.mark.parametrize("case", range(len(LARGE)))
def test_oracle_matches_reference_on_a_large_lattice(case):
    n, bc, p = LARGE[case]
    ref = need(n)
    u = O.generate_links(n, bc, 300 + case, 0.25)
    ref.set_field(bc, u)
    got = ref.measure(p)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    want, want_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    assert scaled_err(got, want, want_abs) <= 1e-13


def test_reference_reproduces_c1_fixture():
    """The 8^4 workload's golden fixture (made by the oracle) reproduced by
    the reference itself."""
    import os
    f = dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                  "c1_8x8x8x8_periodic.npz")))
    n = tuple(int(x) for x in f["n"])
    ref = need(n)
    p = WloopParms(msl=int(f["msl"]), nss=[int(x) for x in f["nss"]], mwlt=int(f["mwlt"]),
                   mwlr=int(f["mwlr"]), alpha_ape=float(f["alpha_ape"]),
                   alpha_action=tuple(f["alpha_action"]), proj_iter=int(f["proj_iter"]))
    ref.set_field(int(f["bc"]), O.generate_links(n, int(f["bc"]), int(f["seed"]),
                                                 float(f["eps"])))
    got = ref.measure(p).reshape(n[0], -1)[f["x0"]]
    assert scaled_err(got, f["wl"], f["wl_abs"]) <= 1e-13


# ---------------------------------------------------------------------------
# GPU against the reference
# ---------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("form", [0, 11])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_gpu_matches_reference(case, form):
    """The default form (the carried lines on these small lattices) and the
    temporal-gauge form (11) against the reference."""
    from wloop_b200 import Context
    n, bc, p = CASES[case]
    ref = need(n)
    u = O.generate_links(n, bc, 200 + case, 0.25)
    ref.set_field(bc, u)
    want = ref.measure(p)
    # |terms| scale of every entry, from the oracle on the same field
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    _, want_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    with Context(n, bc, "fp64") as c:
        c.set_contract_tuning(variant=form)
        c.upload(u)
        got = c.measure(p)
    err = scaled_err(got, want, want_abs)
    nz = want != 0.0
    rel = np.abs(got - want)[nz] / np.abs(want)[nz]
    print(f"fp64 vs reference: max scaled {err:.2e}, max plain relative {rel.max():.2e}")
    assert err <= 1e-12
    assert rel.max() <= 1e-12  # these fields hold no near-zero W
    with Context(n, bc, "mixed") as c:
        c.set_contract_tuning(variant=form)
        c.upload(u)
        gm = c.measure(p)
    assert np.all(gm[~nz] == 0.0)
    relm = np.abs(gm - want)[nz] / np.abs(want)[nz]
    print(f"mixed vs reference: max plain relative {relm.max():.2e}")
    assert relm.max() <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("case", range(len(LARGE)))
def test_gpu_default_form_matches_reference_on_a_large_lattice(case):
    """32x16^3 (131,072 sites): a context's default there is the temporal
    gauge form; against the reference itself, both precisions."""
    from wloop_b200 import Context
    n, bc, p = LARGE[case]
    ref = need(n)
    u = O.generate_links(n, bc, 400 + case, 0.25)
    ref.set_field(bc, u)
    want = ref.measure(p)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    _, want_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    nz = want != 0.0
    for prec in ("fp64", "mixed"):
        with Context(n, bc, prec) as c:
            c.upload(u)
            got = c.measure(p)
            assert c.contract_form == 11
        assert np.all(got[~nz] == 0.0)
        rel = np.abs(got - want)[nz] / np.abs(want)[nz]
        print(f"{prec} vs reference: max plain relative {rel.max():.2e}")
        if prec == "fp64":
            assert scaled_err(got, want, want_abs) <= 1e-12
        else:
            assert rel.max() <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("bc", [0, 3])
def test_gpu_smearing_and_plaquette_match_reference(bc):
    from wloop_b200 import Context
    n = (8, 8, 8, 8)
    ref = need(n)
    u = O.generate_links(n, bc, 300 + bc, 0.3)
    ref.set_field(bc, u)
    ref.hyp_links(1.0, 1.0, 0.5, 1, 4)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        c.hyp_links(1.0, 1.0, 0.5, 1, 4)
        assert np.abs(c.download() - ref.get_field()).max() < 1e-13
        p0 = c.lnk_plaq_sum()
        assert abs(p0 - ref.plaq_sum()) <= 1e-13 * abs(p0)
        c.ape_spatial_links(0.5, 1, 4, nsweeps=4)
        ref.ape_links(0.5, 1, 4, time=0, nsweeps=4)
        assert np.abs(c.download() - ref.get_field()).max() < 1e-13
