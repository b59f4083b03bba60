"""An exact integer form of the temporal-gauge Gram product, checked on the
CPU against the oracle.

Every element x of the transformed lines, divided by a fixed power-of-two
bound S = 2 (entries of products of near-unitary matrices stay below about
1.6 while |g g^dag - 1| <= 1/4, the form's eligibility rule), is written as
s signed 7-bit slices, x ~ S sum_i q_i 2^(-7(i+1)) with |q_i| <= 127 (each
slice the rounded remainder of the ones before), and

    W = S^2 sum over slice pairs (i, j), i + j <= m, of 2^(-7(i+j+2)) (q_A,i . q_B,j).

The slice-pair dot products are exact integers (on the tensor cores an int8
MMA with 32-bit accumulation: every partial sum here stays below 2^31) and
are combined in FP64 in a fixed order, so a device form can reproduce this
restatement bit for bit. On lines rounded to FP32 (the mixed form's lines)
3 slices and 6 pairs keep W within the mixed bar of the oracle (1.3-1.6e-7
plain relative on these 4^3 lattices; the slicing error of W shrinks as
more columns are summed) and 4 slices and 10 pairs within 1e-8 of the
exact product of the same lines; 7 slices and 28 pairs on FP64 lines keep
it within the FP64 bar.
"""
import numpy as np
import pytest

from tests import oracle as O
from tests.test_temporal_gauge import CASES, banded_gram, transformed_lines

S = 2.0


def slice_rows(v, s):
    r = v / S
    qs = []
    for i in range(s):
        q = np.rint(r * 2.0 ** (7 * (i + 1)))
        assert np.abs(q).max() <= 127
        qs.append(q.astype(np.int64))
        r = r - q * 2.0 ** (-7 * (i + 1))
    return qs


def sliced_dot(s, m):
    pairs = sorted(((i, j) for i in range(s) for j in range(s) if i + j <= m),
                   key=lambda t: (t[0] + t[1], t[0]))

    def dot(va, vb):  # va, vb: [levels][columns]
        qa, qb = slice_rows(va, s), slice_rows(vb, s)
        w = np.zeros((va.shape[0], vb.shape[0]))
        for i, j in pairs:
            d = qa[i] @ qb[j].T  # exact
            assert np.abs(np.cumsum(qa[i][:, None, :] * qb[j][None, :, :], axis=-1)).max() < 2**31
            w += d.astype(np.float64) * 2.0 ** (-7 * (i + j + 2))
        return w * (S * S)
    return dot


PROJECTED = [c for c in range(len(CASES)) if CASES[c][2].proj_iter >= 3]


@pytest.mark.parametrize("case", PROJECTED)
def test_int8_slices_reproduce_the_oracle(case):
    n, bc, p = CASES[case]
    u = O.generate_links(n, bc, 70 + case, 0.3)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    want, want_abs, levels = O.wloop_sum(n, bc, uh, p, want_abs=True, want_levels=True)
    zero = want == 0.0

    def lines32():
        for R, va, vb in transformed_lines(n, bc, uh, levels, p):
            yield R, va.astype(np.float32).astype(np.float64), vb.astype(np.float32).astype(np.float64)

    mixed = banded_gram(n, bc, p, lines32(), sliced_dot(3, 2))
    assert np.array_equal(mixed[zero], want[zero])
    rel = np.abs(mixed - want)[~zero] / np.abs(want)[~zero]
    print(f"3 slices, 6 pairs on FP32 lines: max plain relative {rel.max():.1e}")
    assert rel.max() <= 1e-6
    exact = banded_gram(n, bc, p, lines32())
    four = banded_gram(n, bc, p, lines32(), sliced_dot(4, 3))
    rel = np.abs(four - exact)[~zero] / np.abs(exact)[~zero]
    print(f"4 slices, 10 pairs against the exact product of the FP32 lines: {rel.max():.1e}")
    assert rel.max() <= 1e-8

    fp64 = banded_gram(n, bc, p, transformed_lines(n, bc, uh, levels, p), sliced_dot(7, 6))
    assert np.array_equal(fp64[zero], want[zero])
    err = np.abs(fp64 - want)[~zero] / np.maximum(np.abs(want), want_abs)[~zero]
    print(f"7 slices, 28 pairs on FP64 lines: max scaled {err.max():.1e}")
    assert err.max() < 1e-13
