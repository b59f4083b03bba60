"""The identity the temporal-gauge contraction rests on, checked on the CPU.

Every term of the loop sum, Re tr[S_s1(x) L_T(x+Rk) S_s2(x+T)^dag L_T(x)^dag]
(wloop.c:436-508), is a closed loop.  With g(x0, xs) = U0(0, xs) ... U0(x0-1, xs)
the temporal line is L_T(x) = g(x0)^-1 g(x0+T) exactly, whether or not the
smeared links are exactly unitary, and the term is the dot product of the 18
real numbers of
    A(x0) = H(x0)^-1 B(x0) H(x0+Rk)^-1   and   B(x0+T),
    B(x)  = g(x) S(x) g(x+Rk)^dag,  H = g g^dag
(A = B when the links are unitary).  For periodic time the time axis is
unrolled to N0 + mwlt slices (g(N0+y) = P g(y)); for open time the loops
through the last slice are exact zeros.  Here that restatement, in numpy on
the oracle's own smearing levels, reproduces the oracle's Wilson loops: the
device form in wloop_b200/csrc/gram.cu computes the same quantity.  The
approximate SU(3) projection leaves the smeared links unitary only to about
1e-8 (4 iterations, smooth fields), so the factors H^-1 are needed for FP64
agreement.
"""
import numpy as np
import pytest

from tests import oracle as O
from wloop_b200.api import APE, HYP, WloopParms


def transformed_lines(n, bc, u, levels, p):
    """Per spatial extent R = 1..mwlr: (R, VA, VB), the A lines of the N0
    start slices and the B lines of the Nu unrolled slices as rows
    [slice][level][column], column = (direction, site, 18 reals)."""
    N0 = n[0]
    ns = np.array(n[1:])
    vs = int(np.prod(ns))
    msl, mwlt, mwlr = p.msl, p.mwlt, p.mwlr
    f = u.reshape(N0, vs, 4, 3, 3)
    Nu = N0 + (0 if bc == 0 else mwlt)
    g = np.empty((Nu, vs, 3, 3), dtype=np.complex128)
    g[0] = np.eye(3)
    for y in range(Nu - 1):
        g[y + 1] = g[y] @ f[y % N0, :, 0]
    xs = np.indices(tuple(ns)).reshape(3, -1).T
    st = np.array([ns[1] * ns[2], ns[2], 1])

    def shifted(k, d):  # spatial index of xs + d k-hat
        y = xs.copy()
        y[:, k] = (y[:, k] + d) % ns[k]
        return y @ st

    lev = levels.reshape(msl, N0, vs, 3, 3, 3)[:, np.arange(Nu) % N0]  # [sl][y][xs][k]
    dag = lambda m: np.conj(np.swapaxes(m, -1, -2))
    hinv = np.linalg.inv(g @ dag(g))
    b = np.empty((msl, 3, Nu, vs, 3, 3), dtype=np.complex128)  # B lines, length 1
    uh = np.empty_like(b)  # recursion links H^-1 B1
    for k in range(3):
        b[:, k] = g[None] @ lev[:, :, :, k] @ dag(g[:, shifted(k, 1)])[None]
        uh[:, k] = hinv[None] @ b[:, k]
    a = np.empty((msl, 3, N0, vs, 3, 3), dtype=np.complex128)

    def rows(m, ny):
        v = m.view(np.float64).reshape(msl, 3, ny, vs * 18)
        return np.transpose(v, (2, 0, 1, 3)).reshape(ny, msl, 3 * vs * 18)  # (slice, level)

    for r in range(mwlr):
        R = r + 1
        for k in range(3):
            if r > 0:
                b[:, k] = b[:, k] @ uh[:, k][:, :, shifted(k, r)]
            a[:, k] = hinv[None, :N0] @ b[:, k, :N0] @ hinv[None, :N0][:, :, shifted(k, R)]
        yield R, rows(a, N0), rows(b, Nu)


def banded_gram(n, bc, p, lines, dot=lambda va, vb: va @ vb.T):
    """wl_mat (wl_idx order) from the transformed lines: W(x0, T) =
    dot(VA[x0], VB[x0 + T]) / (9 N1 N2 N3); loops through the last slice of
    open time are exact zeros."""
    N0, msl, mwlt, mwlr = n[0], p.msl, p.mwlt, p.mwlr
    norm = 9.0 * n[1] * n[2] * n[3]
    wl = np.zeros(N0 * mwlr * mwlt * msl * msl)
    for R, va, vb in lines:
        r = R - 1
        for x0 in range(N0):
            for T in range(1, mwlt + 1):
                if bc == 0 and x0 + T >= N0:
                    continue  # through the zero temporal link of the last slice
                w = dot(va[x0], vb[x0 + T]) / norm  # [s1][s2]
                for s1 in range(msl):
                    for s2 in range(msl):
                        wl[s1 + msl * (s2 + msl * (T - 1 + mwlt * (r + mwlr * x0)))] = w[s1, s2]
    return wl


def temporal_gauge_wloops(n, bc, u, levels, p):
    return banded_gram(n, bc, p, transformed_lines(n, bc, u, levels, p))


CASES = [
    ((8, 4, 4, 4), 3, WloopParms(msl=3, nss=[0, 2, 2], mwlt=5, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((8, 4, 4, 4), 0, WloopParms(msl=3, nss=[0, 2, 2], mwlt=5, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((6, 4, 6, 2), 3, WloopParms(msl=2, nss=[1, 1], mwlt=4, mwlr=2, op_smear=HYP,
                                 alpha_hyp=(0.75, 0.3), proj_iter=3)),
    ((6, 4, 4, 4), 3, WloopParms(msl=2, nss=[0, 1], mwlt=4, mwlr=2, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=2)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_temporal_gauge_gram_equals_oracle(case):
    n, bc, p = CASES[case]
    u = O.generate_links(n, bc, 70 + case, 0.3)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    want, want_abs, levels = O.wloop_sum(n, bc, uh, p, want_abs=True, want_levels=True)
    got = temporal_gauge_wloops(n, bc, uh, levels, p)
    zero = want == 0.0
    assert np.array_equal(got[zero], want[zero])
    if bc == 0:
        assert zero.any()  # the crossing loops exist and are exact zeros
    err = np.abs(got - want)[~zero] / np.maximum(np.abs(want), want_abs)[~zero]
    assert err.max() < 1e-13
