"""Exact symmetries of the measurement, checked on the device at small and at
full size (the reference's devel/wloop/check2.c and check3.c).

* The device gauge transformation and translation equal their numpy
  definitions on the host (bit-exact for the translation, a permutation).
* A random gauge transformation leaves every W(sl1,sl2;t,r;x0) unchanged and
  a translation by s moves it to x0 - s0, within the reference's tolerances
  |1 - W'/W| < 100 sqrt(msl^2 mwlr mwlt 3 V) DBL_EPSILON (gauge) and
  100 sqrt(1296 msl^2 mwlr mwlt 3 V) DBL_EPSILON (translation), in FP64; the
  mixed form is held to the same bounds or 1e-6, whichever is larger.
* At 32^3x64 (the bench workload) the same holds for both forms: the
  full-size parity evidence that needs no CPU reference.
"""
import math

import numpy as np
import pytest

from wloop_b200 import APE, HYP, Context, WloopParms, generate_links
from wloop_b200.workloads import C3

pytestmark = pytest.mark.gpu

DBL_EPS = np.finfo(np.float64).eps


def tol_gauge(p, vol):
    return 100 * math.sqrt(p.msl * p.msl * p.mwlr * p.mwlt * 3 * vol) * DBL_EPS


def tol_shift(p, vol):
    return 100 * math.sqrt(1296 * p.msl * p.msl * p.mwlr * p.mwlt * 3 * vol) * DBL_EPS


def rel_dev(a, b):
    nz = b != 0.0
    assert np.all(a[~nz] == 0.0), "a loop that vanishes in one measurement must vanish in both"
    return float(np.max(np.abs(1.0 - a[nz] / b[nz]))) if nz.any() else 0.0


def host_gauge(u, n, seed, eps):
    """U_mu(x) -> g(x) U_mu(x) g(x+mu)^dag with g(x) = generated link number x."""
    vol = u.shape[0]
    gfield = generate_links(n, 3, seed, eps).reshape(4 * vol, 3, 3)[:vol]
    x = np.indices(n).reshape(4, -1).T  # lexicographic order, x3 fastest
    st = np.array([n[1] * n[2] * n[3], n[2] * n[3], n[3], 1])
    out = np.empty_like(u)
    for mu in range(4):
        y = x.copy()
        y[:, mu] = (y[:, mu] + 1) % n[mu]
        gy = gfield[y @ st]
        out[:, mu] = gfield @ u[:, mu] @ np.conj(np.transpose(gy, (0, 2, 1)))
    return out


def host_shift(u, n, s):
    f = u.reshape(*n, 4, 3, 3)
    return np.roll(f, shift=tuple(s), axis=(0, 1, 2, 3)).reshape(u.shape)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_device_transforms_match_definitions(prec):
    n = (6, 4, 6, 8)
    u = generate_links(n, 3, 31, 0.3)
    with Context(n, 3, prec) as c:
        c.upload(u)
        c.gauge_transform(77, 0.8)
        got = c.download()
        c.upload(u)
        c.shift_ud((1, -2, 3, 5))
        sh = c.download()
    want = host_gauge(u, n, 77, 0.8)
    tol = 1e-13 if prec == "fp64" else 2e-6
    assert np.max(np.abs(got - want)) < tol
    want_sh = host_shift(u, n, (1, -2, 3, 5))
    if prec == "fp64":
        assert np.array_equal(sh, want_sh)
    else:  # the FP32 field is a permutation of the rounded input
        with Context(n, 3, prec) as c:
            c.upload(u)
            r = c.download()
        assert np.array_equal(sh, host_shift(r, n, (1, -2, 3, 5)))


def test_shift_rejects_time_shift_with_open_bc():
    n = (6, 4, 4, 4)
    with Context(n, 0, "fp64") as c:
        c.generate(1, 0.2)
        with pytest.raises(Exception, match="spatial shifts only"):
            c.shift_ud((1, 0, 0, 0))
        c.shift_ud((0, 1, 0, 2))


def _measure_pair(n, bc, prec, p, seed, eps, transform):
    with Context(n, bc, prec) as c:
        c.generate(seed, eps)
        c.snapshot()
        w0 = c.measure(p)
        c.restore()
        transform(c)
        w1 = c.measure(p)
    return w0, w1


CASES = [
    ((8, 4, 4, 4), 3, WloopParms(msl=3, nss=[0, 1, 2], mwlt=4, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((8, 6, 4, 4), 0, WloopParms(msl=2, nss=[1, 2], mwlt=4, mwlr=2, op_smear=HYP,
                                 alpha_hyp=(0.75, 0.3), proj_iter=3)),
]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_gauge_invariance_small(case, prec):
    n, bc, p = CASES[case]
    vol = int(np.prod(n))
    w0, w1 = _measure_pair(n, bc, prec, p, 5, 0.25, lambda c: c.gauge_transform(123, 1.0))
    tol = tol_gauge(p, vol) if prec == "fp64" else max(tol_gauge(p, vol), 1e-6)
    assert rel_dev(w1, w0) < tol


@pytest.mark.parametrize("case", range(len(CASES)))
def test_translation_small(case):
    n, bc, p = CASES[case]
    vol = int(np.prod(n))
    block = p.msl * p.msl * p.mwlr * p.mwlt
    shifts = [(0, 1, 0, -1), (0, 0, -1, 1)] + ([(1, 0, 1, 0), (-1, 1, 0, 0)] if bc == 3 else [])
    for s in shifts:
        w0, w1 = _measure_pair(n, bc, "fp64", p, 9, 0.25, lambda c: c.shift_ud(s))
        want = np.roll(w0, s[0] * block)  # W'(x0) = W(x0 - s0), x0 slowest
        assert rel_dev(w1, want) < tol_shift(p, vol), s


@pytest.mark.parametrize("prec", ["mixed", "fp64"])
def test_full_size_invariances(prec):
    """32^3x64, HYP2 + 6 APE levels, msl 6, r <= 16, t <= 24 (the bench
    workload): gauge invariance and a translation by (1,0,-1,1)."""
    w = C3
    p = w.parms
    vol = w.volume
    block = p.msl * p.msl * p.mwlr * p.mwlt
    with Context(w.n, w.bc, prec) as c:
        c.generate(w.seed, w.eps)
        c.snapshot()
        w0 = c.measure(p)
        c.restore()
        c.gauge_transform(4242, 1.0)
        wg = c.measure(p)
        c.restore()
        c.shift_ud((1, 0, -1, 1))
        ws = c.measure(p)
    tg = tol_gauge(p, vol) if prec == "fp64" else max(tol_gauge(p, vol), 1e-6)
    ts = tol_shift(p, vol) if prec == "fp64" else max(tol_shift(p, vol), 1e-6)
    assert rel_dev(wg, w0) < tg
    assert rel_dev(ws, np.roll(w0, block)) < ts


def test_bounded_wait_ends():
    """The bounded wait of the bulk-staged contraction, on a barrier that no
    copy completes: it ends at its limit and reports, and the device stays
    usable for the next measurement."""
    import ctypes as C
    from wloop_b200._native import lib
    out, el = C.c_int(-1), C.c_double(-1.0)
    assert lib.wlg_selftest_wait(0, 0.2, C.byref(out), C.byref(el)) == 0
    assert out.value == 1
    assert 0.2 <= el.value < 2.0
    n, bc, p = CASES[0]
    with Context(n, bc, "fp64") as c:
        c.generate(3, 0.2)
        c.set_contract_tuning(7, 3, 0, 0, 64)
        w1 = c.measure(p)
    assert np.all(np.isfinite(w1))


def test_largest_serving_volume_invariances():
    """48^3x96 with open boundary conditions, the largest lattice of the
    serving mix (HYP2 + 4 APE levels, msl 4, r,t <= 24), mixed form: gauge
    invariance and a spatial translation by (0,1,-1,2), which leaves every
    per-slice W unchanged."""
    from wloop_b200.workloads import SERVE_VOLUMES, serving_request
    n = SERVE_VOLUMES[-1]
    w = next(serving_request(i) for i in range(1000) if serving_request(i).n == n)
    p = w.parms
    vol = int(np.prod(n))
    with Context(n, 0, "mixed") as c:
        c.generate(w.seed, w.eps)
        c.snapshot()
        w0 = c.measure(p)
        c.restore()
        c.gauge_transform(99, 1.0)
        wg = c.measure(p)
        c.restore()
        c.shift_ud((0, 1, -1, 2))
        ws = c.measure(p)
    assert rel_dev(wg, w0) < max(tol_gauge(p, vol), 1e-6)
    assert rel_dev(ws, w0) < max(tol_shift(p, vol), 1e-6)
