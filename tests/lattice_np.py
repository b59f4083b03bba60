"""numpy helpers for the tests: direct (definition-level) restatements used
to cross-check the oracle's bookkeeping, plus gauge transformations and
lattice shifts used by the reference's invariance checks
(devel/wloop/check2.c, devel/wloop/check3.c).

Fields are complex arrays of shape (V, 4, 3, 3) in lexicographic order
(x3 fastest); as5d() views them as [x0, x1, x2, x3, mu, 3, 3].
"""
import numpy as np


def as5d(u, n):
    return u.reshape(n[0], n[1], n[2], n[3], 4, 3, 3)


def dag(a):
    return np.conj(np.swapaxes(a, -1, -2))


def mm(a, b):
    return np.matmul(a, b)


def unit_field(n, bc):
    u = np.zeros((int(np.prod(n)), 4, 3, 3), dtype=np.complex128)
    u[:] = np.eye(3)
    if bc == 0:
        as5d(u, n)[n[0] - 1, :, :, :, 0] = 0.0
    return u


def random_su3(shape, rng):
    """Haar-like random SU(3) matrices (QR of complex Gaussians, det fixed)."""
    z = (rng.standard_normal(shape + (3, 3)) + 1j * rng.standard_normal(shape + (3, 3))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    d = np.diagonal(r, axis1=-2, axis2=-1)
    q = q * (d / np.abs(d))[..., None, :]
    det = np.linalg.det(q)
    q = q / (det ** (1.0 / 3.0))[..., None, None]
    return q


def gauge_transform(u, n, bc, g):
    """U'(x,mu) = g(x) U(x,mu) g(x+mu)^dag; g has shape (N0,N1,N2,N3,3,3).
    With open bc the zero temporal links at x0=N0-1 stay zero."""
    U = as5d(u, n)
    out = np.empty_like(U)
    for mu in range(4):
        gp = np.roll(g, -1, axis=mu)
        out[..., mu, :, :] = mm(mm(g, U[..., mu, :, :]), dag(gp))
    if bc == 0:
        out[n[0] - 1, :, :, :, 0] = 0.0
    return out.reshape(u.shape)


def shift_field(u, n, s):
    """Translate the field: U'(x) = U(x - s) (openQCD shift_ud convention is
    irrelevant here; the test only needs a consistent x0 bookkeeping)."""
    U = as5d(u, n)
    out = np.roll(U, shift=tuple(s), axis=(0, 1, 2, 3))
    return out.reshape(u.shape)


def plaq_sum(u, n, bc):
    """Sum over plaquettes of Re tr U(p) (lnkplaq.c:48-114 definition)."""
    U = as5d(u, n)
    tot = 0.0
    for mu in range(1, 4):
        for nu in range(0, mu):
            a = mm(U[..., mu, :, :], np.roll(U[..., nu, :, :], -1, axis=mu))
            b = mm(U[..., nu, :, :], np.roll(U[..., mu, :, :], -1, axis=nu))
            tr = np.real(np.sum(np.conj(a) * b, axis=(-1, -2)))
            if nu == 0 and bc == 0:
                tr = tr[: n[0] - 1]
            tot += tr.sum()
    return tot


def staple_sum(u1, u2, n, mu, nu):
    """up + down staples of the (mu,nu) plane (lnkstaple.c:43-56)."""
    A = as5d(u1, n)[..., nu, :, :]
    B = as5d(u2, n)[..., mu, :, :]
    up = mm(mm(A, np.roll(B, -1, axis=nu)), dag(np.roll(A, -1, axis=mu)))
    An = np.roll(A, 1, axis=nu)
    Bn = np.roll(B, 1, axis=nu)
    An_pm = np.roll(An, -1, axis=mu)
    dn = mm(mm(dag(An), Bn), An_pm)
    return (up + dn).reshape(-1, 3, 3)


def wloops_direct(u0field, levels, n, msl, mwlt, mwlr):
    """Definition of W(sl1,sl2;t,r;x0) (README.ms10 'OUTPUT DATA', wloop.c:476-487):
    1/(9 N1 N2 N3) sum_{xs,k} Re tr[(ub um)^dag (ul ubR)] with ub, ubR temporal
    lines of length T at x and x+R k, ul, um spatial lines of length R of level
    sl1 at x and sl2 at x+T 0.  Returns array [x0, r, t, sl2, sl1]."""
    U = as5d(u0field, n)
    U0 = U[..., 0, :, :]
    lv = [levels[s].reshape(n[0], n[1], n[2], n[3], 3, 3, 3) for s in range(msl)]
    out = np.zeros((n[0], mwlr, mwlt, msl, msl))
    norm = 9.0 * n[1] * n[2] * n[3]
    for r in range(mwlr):
        R = r + 1
        lines = []
        for s in range(msl):
            per_k = []
            for k in range(3):
                Uk = lv[s][..., k, :, :]
                L = Uk.copy()
                for j in range(1, R):
                    L = mm(L, np.roll(Uk, -j, axis=k + 1))
                per_k.append(L)
            lines.append(per_k)
        LT = U0.copy()
        for t in range(mwlt):
            T = t + 1
            if T > 1:
                LT = mm(LT, np.roll(U0, -(T - 1), axis=0))
            for k in range(3):
                ubR = np.roll(LT, -R, axis=k + 1)
                for s1 in range(msl):
                    ul = lines[s1][k]
                    B = mm(ul, ubR)
                    for s2 in range(msl):
                        um = np.roll(lines[s2][k], -T, axis=0)
                        A = mm(LT, um)
                        tr = np.real(np.sum(np.conj(A) * B, axis=(-1, -2)))
                        out[:, r, t, s2, s1] += tr.sum(axis=(1, 2, 3))
    return out / norm
