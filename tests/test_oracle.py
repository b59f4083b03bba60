"""CPU tests of the FP64 oracle against the reference's own checks.

The reference ships no golden vectors (devel/smear/check1.c needs the
missing 8x8x8x8_cnfg files), so the oracle is pinned by the properties its
devel/ programs assert, restated here, plus an independent definition-level
numpy restatement of the loop sums:
  * projection: unitarity and det = 1 after projection (devel/smear/check2.c)
  * hyp_links(a,0,0) == (1-a) ape_links(a/6/(1-a)) and the spatial analogue
    (devel/smear/check3.c:92-189), for open and periodic bc
  * unit field: every W = 1, loops crossing an open boundary 0
    (devel/wloop/check1.c:85-122, input check1.in)
  * gauge invariance of HYP + smearing + loops (devel/wloop/check2.c:255-372)
  * translation invariance (devel/wloop/check3.c:87-153)
  * staple and plaquette definitions (devel/lnk/check1.c, check2.c)
"""
import numpy as np
import pytest

from tests import lattice_np as L
from tests import oracle as O
from wloop_b200.api import APE, HYP, WloopParms, generate_links

DBL_EPS = np.finfo(float).eps


def rnd_field(n, bc, seed=7, eps=0.3):
    return generate_links(n, bc, seed, eps)


def test_projection_unitarity_and_det():
    rng = np.random.default_rng(1)
    m = rng.standard_normal((50, 3, 3)) + 1j * rng.standard_normal((50, 3, 3))
    m = m * 0.3 + np.eye(3)
    p = O.project(m, 30)
    dev_u = np.abs(p @ L.dag(p) - np.eye(3)).max()
    dev_d = np.abs(np.linalg.det(p) - 1).max()
    assert dev_u < 1e-13 and dev_d < 1e-13
    # SU(3) input is a fixed point (to rounding)
    su3 = L.random_su3((20,), rng)
    assert np.abs(O.project(su3, 4) - su3).max() < 1e-14


def test_projection_zero_guard():
    z = np.zeros((1, 3, 3), dtype=np.complex128)
    assert np.all(O.project(z, 5) == 0)  # projection.c:136


@pytest.mark.parametrize("n", [(4, 4, 4, 4), (4, 2, 4, 6)])
def test_staple_sum_definition(n):
    u1 = rnd_field(n, 3, seed=3)
    u2 = rnd_field(n, 3, seed=4)
    vb0 = rnd_field(n, 3, seed=5)
    for mu, nu in [(0, 1), (2, 0), (3, 2), (1, 3)]:
        got = O.staple_sum(n, u1, u2, mu, nu, vb0)
        exp = vb0.copy()
        exp[:, mu] += L.staple_sum(u1, u2, n, mu, nu)
        assert np.abs(got - exp).max() < 1e-14


@pytest.mark.parametrize("bc", [0, 3])
def test_plaquette_definition(bc):
    n = (4, 4, 2, 6)
    u = rnd_field(n, bc, seed=11)
    assert abs(O.plaq_sum(n, bc, u) - L.plaq_sum(u, n, bc)) < 1e-11


@pytest.mark.parametrize("bc", [0, 3])
def test_unit_field_plaquette(bc):
    n = (4, 4, 4, 4)
    u = L.unit_field(n, bc)
    v = np.prod(n)
    nplaq = (6 * n[0] - 3) * v // n[0] if bc == 0 else 6 * v  # devel/smear/check3.c:85-88
    assert O.plaq_sum(n, bc, u) == pytest.approx(3.0 * nplaq, rel=1e-15)


@pytest.mark.parametrize("bc", [0, 3])
def test_hyp_ape_identity(bc):
    """devel/smear/check3.c: hyp_links(a,0,0,no proj) == (1-a) ape_links(a/6/(1-a))."""
    n = (4, 4, 4, 4)
    u = rnd_field(n, bc, seed=21)
    alpha = 0.5
    a = 1.0 - alpha
    uh = O.hyp_links(n, bc, u, alpha, 0.0, 0.0, 0, 0)
    ua = O.ape_links(n, u, alpha / 6.0 / a, 0, 0, time=1)
    assert np.abs(uh - a * ua).max() < 1e-14
    p1, p2 = O.plaq_sum(n, bc, uh), O.plaq_sum(n, bc, ua)
    assert abs(p1 - a ** 4 * p2) / (6 * np.prod(n)) < 1e-14
    # spatial form: temporal links untouched
    us = O.hyp_spatial_links(n, u, alpha, 0.0, 0, 0)
    ua = O.ape_links(n, u, alpha / 4.0 / a, 0, 0, time=0)
    assert np.abs(us[:, 0] - u[:, 0]).max() == 0.0
    assert np.abs(us[:, 1:] - a * ua[:, 1:]).max() < 1e-14


def test_hyp_projected_is_su3():
    """devel/smear/check2.c: after hyp_links with projection the links are near SU(3)."""
    n = (4, 4, 4, 4)
    u = rnd_field(n, 3, seed=5)
    uh = O.hyp_links(n, 3, u, 0.75, 0.6, 0.3, 1, 30)
    m = uh.reshape(-1, 3, 3)
    assert np.abs(m @ L.dag(m) - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(m) - 1).max() < 1e-12


def test_hyp_masks():
    """hyp_time_links / hyp_space_links only replace their directions."""
    n = (4, 4, 4, 4)
    u = rnd_field(n, 3, seed=8)
    full = O.hyp_links(n, 3, u, 1.0, 1.0, 0.5, 1, 4)
    t = O.hyp_links(n, 3, u, 1.0, 1.0, 0.5, 1, 4, time=1, space=0)
    s = O.hyp_links(n, 3, u, 1.0, 1.0, 0.5, 1, 4, time=0, space=1)
    assert np.array_equal(t[:, 0], full[:, 0]) and np.array_equal(t[:, 1:], u[:, 1:])
    assert np.array_equal(s[:, 1:], full[:, 1:]) and np.array_equal(s[:, 0], u[:, 0])


@pytest.mark.parametrize("bc", [0, 3])
def test_unit_field_wloops(bc):
    """devel/wloop/check1.c with check1.in (APE 0.5, nss 0 1 2 3, proj 10)."""
    n = (8, 4, 4, 4)
    u = L.unit_field(n, bc)
    u = O.hyp_links(n, bc, u, 1.0, 1.0, 0.5, 1, 10, time=1, space=0)
    p = WloopParms(msl=4, nss=[0, 1, 2, 3], mwlt=4, mwlr=3, op_smear=APE, alpha_ape=0.5,
                   proj_iter=10)
    wl = O.wloop_sum(n, bc, u, p).reshape(n[0], p.mwlr, p.mwlt, p.msl, p.msl)
    eps = np.sqrt(3.0) * n[0] * n[1] / 4 * DBL_EPS
    for x0 in range(n[0]):
        for t in range(p.mwlt):
            crosses = bc == 0 and x0 + t + 1 > n[0] - 1
            blk = wl[x0, :, t]
            if crosses:
                assert np.all(blk == 0.0)
            else:
                assert np.abs(blk - 1.0).max() < eps


@pytest.mark.parametrize("bc,op", [(3, APE), (0, APE), (3, HYP), (0, HYP)])
def test_wloops_match_definition(bc, op):
    """Oracle loop bookkeeping (x0 wrap, wl_idx, level order) == direct definition."""
    n = (6, 4, 2, 4)
    u = rnd_field(n, bc, seed=31 + bc)
    u = O.hyp_links(n, bc, u, 1.0, 1.0, 0.5, 1, 4)
    p = WloopParms(msl=3, nss=[0, 1, 2], mwlt=3, mwlr=2, op_smear=op, alpha_ape=0.5,
                   alpha_hyp=(0.75, 0.3), proj_iter=4)
    wl, lv = O.wloop_sum(n, bc, u, p, want_levels=True)
    direct = L.wloops_direct(u, lv, n, p.msl, p.mwlt, p.mwlr)
    got = wl.reshape(n[0], p.mwlr, p.mwlt, p.msl, p.msl)
    assert np.abs(got - direct).max() < 1e-13


@pytest.mark.parametrize("bc", [0, 3])
def test_gauge_invariance(bc):
    """devel/wloop/check2.c with check2.in (HYP 1.0 0.5, proj_iter 0)."""
    n = (4, 4, 4, 4)
    u = rnd_field(n, bc, seed=41)
    p = WloopParms(msl=3, nss=[0, 1, 2], mwlt=3, mwlr=2, op_smear=HYP, alpha_hyp=(1.0, 0.5),
                   proj_iter=0)
    w1 = O.wloop_sum(n, bc, O.hyp_links(n, bc, u, 1.0, 1.0, 0.5, 0, 0), p)
    g = L.random_su3(tuple(n), np.random.default_rng(2))
    ug = L.gauge_transform(u, n, bc, g)
    w2 = O.wloop_sum(n, bc, O.hyp_links(n, bc, ug, 1.0, 1.0, 0.5, 0, 0), p)
    eps = 100 * np.sqrt(p.msl ** 2 * p.mwlr * p.mwlt * 3 * np.prod(n)) * DBL_EPS
    nz = w1 != 0
    assert np.array_equal(w2 == 0, ~nz)
    assert np.abs(1.0 - w2[nz] / w1[nz]).max() < eps


def test_translation_invariance():
    """devel/wloop/check3.c with check3.in (HYP 1.0 0.5, proj_iter 20), periodic."""
    n = (6, 4, 4, 4)
    bc = 3
    u = rnd_field(n, bc, seed=51)
    p = WloopParms(msl=2, nss=[0, 1], mwlt=3, mwlr=2, op_smear=HYP, alpha_hyp=(1.0, 0.5),
                   proj_iter=20)
    w1 = O.wloop_sum(n, bc, O.hyp_links(n, bc, u, 1.0, 1.0, 0.5, 1, 20), p)
    w1 = w1.reshape(n[0], -1)
    eps = 100 * np.sqrt(1296 * p.msl ** 2 * p.mwlr * p.mwlt * 3 * np.prod(n)) * DBL_EPS
    for s in [(1, -1, 0, 0), (0, 1, 0, 1), (-1, 0, 1, 0)]:
        us = L.shift_field(u, n, s)
        w2 = O.wloop_sum(n, bc, O.hyp_links(n, bc, us, 1.0, 1.0, 0.5, 1, 20), p).reshape(n[0], -1)
        w1s = np.roll(w1, s[0], axis=0)
        assert np.abs(1.0 - w2 / w1s).max() < eps


def test_parameter_ranges():
    """set_wloop_parms range checks (wloop_parms.c:156-177)."""
    n = (4, 4, 4, 4)
    u = L.unit_field(n, 3)
    bad = [WloopParms(msl=0, nss=[], mwlt=1, mwlr=1),
           WloopParms(msl=1, nss=[0], mwlt=4, mwlr=1),
           WloopParms(msl=1, nss=[0], mwlt=1, mwlr=4)]
    for p in bad:
        with pytest.raises(ValueError):
            O.wloop_sum(n, 3, u, p)
    ok = WloopParms(msl=1, nss=[0], mwlt=3, mwlr=3)
    O.wloop_sum(n, 3, u, ok)
