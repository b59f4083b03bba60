"""The temporal-gauge contraction form (wloop_b200/csrc/gram.cu) on the GPU.

It is a context's default on lattices of at least 32768 sites and can be
asked for on any (contraction form 11): on the lattices of the parity cases
(odd extents, time slices that are not whole 32-site tiles, 1 to 8 levels,
open and periodic time, the largest loops the parameters allow) it agrees
with the carried-temporal-line form and with the FP64 oracle at the same
bars (FP64: 1e-12 of max(|W|, sum|terms|/norm); mixed: 1e-6 plain
relative), the lattices whose start slices need several blocks and whose
columns are split over several blocks agree as well, and a field smeared
without projection (g far from unitary) falls back to the carried-line form.
"""
import numpy as np
import pytest

from tests import oracle as O
from tests.forms import carried_form
from tests.test_gpu_parity import CASES, assert_wl_close
from wloop_b200 import APE, Context, WloopParms, generate_links

pytestmark = pytest.mark.gpu

PROJECTED = [i for i, (_, _, p) in enumerate(CASES) if p.proj_iter > 0]

# start slices over two blocks (N0 = 40 > the 36 / 23 slices one block of
# 6 levels and mwlt 21 holds), unrolled time 61, several column splits
WIDE = [
    ((40, 4, 4, 4), 3, WloopParms(msl=6, nss=[0, 1, 1, 1, 1, 1], mwlt=21, mwlr=3,
                                  op_smear=APE, alpha_ape=0.5, proj_iter=4)),
    ((40, 4, 4, 4), 0, WloopParms(msl=6, nss=[0, 1, 1, 1, 1, 1], mwlt=21, mwlr=3,
                                  op_smear=APE, alpha_ape=0.5, proj_iter=4)),
    # 7 levels and t <= 49: the rows of one start slice do not fit two stages
    # in half an SM's shared memory, so FP64 takes its one-block-per-SM kernel
    ((96, 4, 4, 4), 3, WloopParms(msl=7, nss=[0, 1, 1, 1, 1, 1, 1], mwlt=49, mwlr=2,
                                  op_smear=APE, alpha_ape=0.5, proj_iter=4)),
    ((96, 4, 4, 4), 0, WloopParms(msl=7, nss=[0, 1, 1, 1, 1, 1, 1], mwlt=49, mwlr=2,
                                  op_smear=APE, alpha_ape=0.5, proj_iter=4)),
]


def _check(prec, got, ref, ref_abs):
    if prec == "fp64":
        assert_wl_close(got, ref, ref_abs)
    else:
        zero = ref == 0.0
        assert np.all(got[zero] == 0.0)
        rel = np.abs(got - ref)[~zero] / np.abs(ref)[~zero]
        print(f"mixed vs oracle: max plain relative {rel.max():.2e}")
        assert rel.max() <= 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", PROJECTED)
def test_form_choice(case, prec):
    """Below 32768 sites the carried lines are the default; form 11 asks for
    the temporal gauge."""
    n, bc, p = CASES[case]
    with Context(n, bc, prec) as c:
        c.generate(900 + case, 0.25)
        c.snapshot()
        c.measure(p)
        assert c.contract_form not in (0, 11)
        c.set_contract_tuning(variant=11)
        c.restore()
        c.measure(p)
        assert c.contract_form == 11


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_default_on_a_large_lattice(prec):
    """16^3x8 (32768 sites) runs the temporal gauge by default and agrees
    with the oracle."""
    n, bc = (8, 16, 16, 16), 3
    p = WloopParms(msl=2, nss=[0, 2], mwlt=4, mwlr=2, op_smear=APE, alpha_ape=0.5, proj_iter=4)
    u = generate_links(n, bc, 960, 0.25)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref, ref_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    with Context(n, bc, prec) as c:
        c.upload(u)
        got = c.measure(p)
        assert c.contract_form == 11
    _check(prec, got, ref, ref_abs)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", [0, 1, 4, 6, 8, 9])
def test_temporal_gauge_against_carried_lines(case, prec):
    n, bc, p = CASES[case]
    u = generate_links(n, bc, 910 + case, 0.25)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref, ref_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    with Context(n, bc, prec) as c:
        c.set_contract_tuning(variant=11)
        c.upload(u)
        c.snapshot()
        gram = c.measure(p)
        assert c.contract_form == 11
        c.set_contract_tuning(variant=carried_form(prec))
        c.restore()
        carried = c.measure(p)
        assert c.contract_form == carried_form(prec)
    _check(prec, gram, ref, ref_abs)
    zero = ref == 0.0
    scale = np.maximum(np.abs(ref), ref_abs)[~zero]
    tol = 2e-12 if prec == "fp64" else 2e-6
    assert np.max(np.abs(gram - carried)[~zero] / scale) <= tol


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("wide", range(len(WIDE)))
def test_several_blocks_and_splits(wide, prec):
    n, bc, p = WIDE[wide]
    u = generate_links(n, bc, 930 + wide, 0.3)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref, ref_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    with Context(n, bc, prec) as c:
        c.set_contract_tuning(variant=11)
        c.upload(u)
        got = c.measure(p)
        assert c.contract_form == 11
        if prec == "fp64" and p.msl == 7:
            assert c.gram_shape(p.msl, p.mwlt)["occ"] == 1
    _check(prec, got, ref, ref_abs)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_unprojected_field_falls_back(prec):
    """Links at 0.85 of the norm of SU(3) matrices, smeared without
    projection (weak HYP weights, so the loops stay of order 1e-4 to 0.3):
    g g^dag is far from 1 already on the second slice (|g g^dag - 1| about
    0.5), so the carried-line form measures (and still agrees with the
    oracle)."""
    n, bc = (8, 4, 4, 4), 3
    p = WloopParms(msl=2, nss=[0, 1], mwlt=4, mwlr=2, op_smear=APE, alpha_ape=0.5, proj_iter=0,
                   alpha_action=(0.2, 0.2, 0.2))
    u = 0.85 * generate_links(n, bc, 940, 0.3)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref, ref_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    with Context(n, bc, prec) as c:
        c.set_contract_tuning(variant=11)  # asked for, not applicable
        c.upload(u)
        got = c.measure(p)
        assert c.contract_form not in (0, 11)
    if prec == "fp64":
        assert_wl_close(got, ref, ref_abs)
    else:
        # loops of shrunken links are small and cancel: scaled bar
        nz = ref != 0.0
        err = np.abs(got - ref)[nz] / np.maximum(np.abs(ref), ref_abs)[nz]
        assert err.max() <= 1e-6


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_kernel_variants_agree_bit_for_bit(prec):
    """Occupancy, FMA order, start slices per block and pipeline depth change
    neither the FMAs of a sum nor their order: the results are identical
    (for a fixed number of column chunks per block)."""
    n, bc, p = WIDE[0]
    with Context(n, bc, prec) as c:
        c.set_contract_tuning(variant=11)
        c.generate(950, 0.3)
        c.snapshot()
        c.set_gram_tuning(cpc=2)
        ref = c.measure(p)
        occs = (1, 2)
        for occ in occs:
            for ord_ in (1, 2):
                for bx, stages in ((0, 0), (8, 2), (13, 3)):
                    c.set_gram_tuning(occ, ord_, bx, stages, 2)
                    try:
                        shape = c.gram_shape(p.msl, p.mwlt)
                    except Exception:
                        continue  # no kernel of this occupancy for this precision and msl
                    c.restore()
                    got = c.measure(p)
                    assert c.contract_form == 11
                    assert np.array_equal(got, ref), (occ, ord_, bx, stages, shape)
