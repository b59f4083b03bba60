"""Batches (wlg_batch): many configurations of different lattices measured
in one CUDA-graph launch must give, configuration by configuration, what one
context gives for each alone (the batched kernels run the same per-lattice
arithmetic and the same reduction order: results are identical), and the
FP64 batch matches the oracle."""
import numpy as np
import pytest

from tests import oracle as O
from wloop_b200 import APE, HYP, Context, WloopParms, generate_links
from wloop_b200.api import Batch
from wloop_b200.autotune import candidates
from wloop_b200.workloads import batch_workloads, flops_per_config

ITEMS = [
    ((8, 4, 4, 4), 3, WloopParms(msl=3, nss=[0, 1, 2], mwlt=3, mwlr=2, op_smear=APE, alpha_ape=0.5,
                                 proj_iter=4)),
    ((6, 4, 6, 4), 0, WloopParms(msl=3, nss=[1, 0, 2], mwlt=3, mwlr=3, op_smear=APE, alpha_ape=0.4,
                                 proj_iter=3)),
    ((8, 6, 4, 4), 3, WloopParms(msl=2, nss=[0, 2], mwlt=4, mwlr=2, op_smear=HYP,
                                 alpha_hyp=(0.75, 0.3), proj_iter=4)),
    ((4, 4, 4, 4), 0, WloopParms(msl=4, nss=[0, 1, 1, 1], mwlt=2, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=0)),
]


def test_batch_workloads_definition():
    ws = batch_workloads()
    assert len(ws) == 64
    assert sum(1 for w in ws if w.n == (32, 16, 16, 16)) == 48
    assert sum(1 for w in ws if w.n == (48, 24, 24, 24)) == 16
    assert all(0.15 <= w.eps <= 0.35 for w in ws)
    assert all(w.parms.mwlr == w.n[1] // 2 and w.parms.mwlt == w.n[1] // 2 for w in ws)
    assert len({w.seed for w in ws}) == 64
    assert flops_per_config(ws[0])["total"] > 0


def test_autotune_candidates():
    assert all(G <= 4 for G, _, _, _ in candidates(4, False, True))
    assert (6, 1, 64, 0) in candidates(6, False, False)
    assert all(G <= 3 and b == 64 for G, SB, b, _ in candidates(6, True, False) if SB != 11)
    # the temporal-gauge form (SB 11) is the first candidate of contexts and batches
    for fp64 in (False, True):
        for batched in (False, True):
            assert candidates(6, fp64, batched)[0] == (0, 11, 0, 0)
    # packed-FMA batch shapes (SB 5) for FP32 batches with unrolled level counts only
    assert any(SB == 5 for _, SB, _, _ in candidates(6, False, True))
    assert not any(SB == 5 for _, SB, _, _ in candidates(6, True, True))
    assert not any(SB == 5 for _, SB, _, _ in candidates(3, False, True))


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_equals_single_contexts(prec):
    fields = [generate_links(n, bc, 300 + i, 0.3) for i, (n, bc, _) in enumerate(ITEMS)]
    singles = []
    for (n, bc, p), u in zip(ITEMS, fields):
        with Context(n, bc, prec) as c:
            c.upload(u)
            singles.append(c.measure(p))
    with Batch(ITEMS, prec) as b:
        for i, u in enumerate(fields):
            b.upload(i, u)
        b.snapshot()
        b.run()
        first = [b.result(i) for i in range(len(ITEMS))]
        b.restore()
        b.run()  # graph replay
        for i in range(len(ITEMS)):
            assert np.array_equal(first[i], singles[i]), f"config {i}"
            assert np.array_equal(b.result(i), singles[i]), f"config {i} (replay)"
        # new field in one slot: only that configuration changes
        u2 = generate_links(ITEMS[1][0], ITEMS[1][1], 999, 0.3)
        b.restore()
        b.upload(1, u2)
        b.run()
        with Context(ITEMS[1][0], ITEMS[1][1], prec) as c:
            c.upload(u2)
            ref1 = c.measure(ITEMS[1][2])
        assert np.array_equal(b.result(1), ref1)
        assert np.array_equal(b.result(0), singles[0])
        ms, kernels = b.stats()
        assert ms > 0 and kernels > 0


@pytest.mark.gpu
def test_batch_fp64_matches_oracle():
    fields = [generate_links(n, bc, 500 + i, 0.25) for i, (n, bc, _) in enumerate(ITEMS)]
    with Batch(ITEMS, "fp64") as b:
        for i, u in enumerate(fields):
            b.upload(i, u)
        b.run()
        for i, ((n, bc, p), u) in enumerate(zip(ITEMS, fields)):
            uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
            ref, ref_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
            got = b.result(i)
            zero = ref == 0.0
            assert np.all(got[zero] == 0.0)
            err = np.abs(got - ref)[~zero] / np.maximum(np.abs(ref), ref_abs)[~zero]
            assert err.max() <= 1e-12


@pytest.mark.gpu
def test_batch_generate_and_shape_change():
    items = ITEMS[:2]
    with Batch(items, "mixed") as b:
        b.generate([7, 8], [0.2, 0.3])
        b.snapshot()
        b.run()
        r0 = [b.result(i) for i in range(2)]
        b.set_contract_shape(G=1, SB=1, nCB=0, block=64)
        b.restore()
        b.run()
        for i in range(2):
            # the third form's FP32 products are not packed like the default's:
            # equal up to FP32 rounding and summation order
            scale = np.maximum(np.abs(r0[i]), 1e-3)
            assert np.max(np.abs(b.result(i) - r0[i]) / scale) < 1e-6
        with Context(items[0][0], items[0][1], "mixed") as c:
            c.generate(7, 0.2)
            assert np.array_equal(c.measure(items[0][2]), r0[0])


# every batched contraction shape (G bottom levels; SB 1, 2: third form, 0:
# fourth form, 3: fourth form with unrolled level loops, 4: fourth form with
# bulk-copy staging, 5: SB 3 with packed FP32 products) gives the batch's
# default result up to summation order, with the line step computed by the
# form that is launched (a stand-alone stage for the third form, inside the
# contraction for the fourth)
BATCH_SHAPES = [(1, 1, 64), (2, 2, 128), (3, 0, 64), (2, 3, 128), (4, 3, 64), (1, 0, 128),
                (3, 4, 64), (2, 4, 128), (4, 5, 64), (3, 5, 128), (1, 5, 32)]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("same_msl", [False, True])
def test_batch_shapes_agree(prec, same_msl):
    items = ITEMS if not same_msl else [
        ((8, 4, 4, 4), 3, WloopParms(msl=4, nss=[0, 1, 1, 2], mwlt=3, mwlr=3, op_smear=APE,
                                     alpha_ape=0.5, proj_iter=4)),
        ((6, 4, 6, 4), 0, WloopParms(msl=4, nss=[1, 0, 2, 1], mwlt=3, mwlr=3, op_smear=APE,
                                     alpha_ape=0.4, proj_iter=3))]
    fields = [generate_links(n, bc, 500 + i, 0.3) for i, (n, bc, _) in enumerate(items)]
    with Batch(items, prec) as b:
        for i, u in enumerate(fields):
            b.upload(i, u)
        b.snapshot()
        b.run()
        ref = [b.result(i) for i in range(len(items))]
        for G, SB, block in BATCH_SHAPES:
            b.set_contract_shape(G=G, SB=SB, nCB=0, block=block)
            b.restore()
            b.run()
            for i in range(len(items)):
                scale = np.maximum(np.abs(ref[i]), 1e-3)
                err = np.max(np.abs(b.result(i) - ref[i]) / scale)
                assert err < (1e-13 if prec == "fp64" else 1e-6), (G, SB, block, i, err)


@pytest.mark.gpu
def test_tune_context_picks_a_shape_with_the_same_result(tmp_path, monkeypatch):
    """The single-context tuner (every candidate, the ninth form among them)
    leaves the context on a shape whose result is the default's up to the
    order of the FP64 sums."""
    from wloop_b200 import autotune
    monkeypatch.setenv("WLG_TUNE_CACHE", str(tmp_path / "tune.json"))
    n, bc = (8, 8, 8, 8), 3
    p = WloopParms(msl=4, nss=[0, 1, 1, 1], mwlt=4, mwlr=3, op_smear=APE, alpha_ape=0.5,
                   proj_iter=4)
    assert any(SB == 9 for _, SB, _, _ in autotune.candidates(4, False, False))
    with Context(n, bc, "mixed") as c:
        c.generate(5, 0.3)
        c.snapshot()
        base = c.measure(p)  # HYP-smears the field in place
        c.restore()  # the tuner snapshots the field it is given
        shape = autotune.tune_context(c, p, "mixed", use_cache=False)
        c.restore()
        got = c.measure(p)
    assert shape in autotune.candidates(4, False, False)
    assert np.abs(got - base).max() <= 1e-6 * np.abs(base).max()


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_batch_temporal_gauge_lattices_equal_contexts(prec):
    """Lattices of at least 32768 sites run the temporal-gauge form in a
    batch as in a context (bit for bit), beside a small lattice that runs the
    carried lines in both."""
    items = [((8, 16, 16, 16), 3, WloopParms(msl=2, nss=[0, 2], mwlt=4, mwlr=3, op_smear=APE,
                                              alpha_ape=0.5, proj_iter=4)),
             ((16, 16, 16, 8), 0, WloopParms(msl=3, nss=[0, 1, 2], mwlt=5, mwlr=2, op_smear=APE,
                                              alpha_ape=0.5, proj_iter=4)),
             ((8, 4, 6, 4), 3, WloopParms(msl=2, nss=[0, 2], mwlt=3, mwlr=2, op_smear=APE,
                                          alpha_ape=0.5, proj_iter=4))]
    fields = [generate_links(n, bc, 970 + i, 0.25) for i, (n, bc, _) in enumerate(items)]
    singles, forms = [], []
    for (n, bc, p), u in zip(items, fields):
        with Context(n, bc, prec) as c:
            c.upload(u)
            singles.append(c.measure(p))
            forms.append(c.contract_form)
    assert forms[0] == 11 and forms[1] == 11 and forms[2] != 11
    with Batch(items, prec) as b:
        for i, u in enumerate(fields):
            b.upload(i, u)
        b.snapshot()
        b.run()
        b.restore()
        b.run()  # graph replay
        for i in range(len(items)):
            assert np.array_equal(b.result(i), singles[i]), f"config {i}"
