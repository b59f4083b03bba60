"""bench.py's reference leg carries its own copy of the workload parameters
(it must not import the product package, whose import loads the CUDA
library); they must stay those of wloop_b200.workloads."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_leg_parameters_match_the_workloads():
    from wloop_b200.workloads import C1, C3
    b = _bench()
    for (n, bc, seed, eps, p), w in (((b.C3_N, b.C3_BC, b.C3_SEED, b.C3_EPS, b.C3_P), C3),
                                      ((b.C1_N, b.C1_BC, b.C1_SEED, b.C1_EPS, b.C1_P), C1)):
        assert tuple(n) == w.n and bc == w.bc and seed == w.seed and eps == w.eps
        q = w.parms
        assert (p.msl, list(p.nss), p.mwlt, p.mwlr) == (q.msl, list(q.nss[:q.msl]), q.mwlt, q.mwlr)
        assert tuple(p.alpha_action) == tuple(q.alpha_action) and p.alpha_ape == q.alpha_ape
        assert p.proj_iter == q.proj_iter and int(p.op_smear) == int(q.op_smear)


def test_loop_piece_is_one_spatial_extent():
    b = _bench()
    for mwlt in (1, 2):
        q = b._loop_piece(b.C3_P, mwlt)
        assert q.mwlr == 1 and q.mwlt == mwlt and q.msl == b.C3_P.msl
        assert list(q.nss) == [0] * q.msl
