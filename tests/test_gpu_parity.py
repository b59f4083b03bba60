"""GPU parity: the sm_100a kernels against the FP64 oracle, through the C ABI.

FP64 bar: every Wilson-loop entry within 1e-12 relative, measured as
|W_gpu - W_oracle| <= 1e-12 * max(|W_oracle|, A_oracle) with A the oracle's
sum of |Re tr| over the averaged terms (entries near zero are limited by
summation order, not by the kernels); the plain relative error is printed
beside it, with every entry above 1e-12 plain listed with its A/|W| ratio.
Entries that are exactly zero in the oracle (loops crossing an open
boundary) must be exactly zero.  Mixed bar: every non-zero entry within 1e-6
plain relative of the FP64 oracle.  Smeared
links and plaquettes: 1e-13 absolute per matrix element / 1e-12 relative.
"""
import numpy as np
import pytest

from tests import lattice_np as L
from tests import oracle as O
from tests.forms import carried_form
from wloop_b200 import APE, HYP, Context, WloopParms, approx_project_to_su3, generate_links
from wloop_b200.api import staple_sum

pytestmark = pytest.mark.gpu

TOL_W = 1e-12


def assert_wl_close(got, ref, ref_abs, tol=TOL_W):
    zero = ref == 0.0
    assert np.all(got[zero] == 0.0), "exact zeros (open-bc crossing loops) must stay exact"
    scale = np.maximum(np.abs(ref), ref_abs)
    diff = np.abs(got - ref)[~zero]
    err = diff / scale[~zero]
    rel = diff / np.abs(ref)[~zero]
    print(f"max scaled error {err.max():.2e}, max plain relative error {rel.max():.2e}")
    # entries above the bar in plain relative terms: each is a near-zero W
    # whose error is set by summation order, i.e. by sum|terms|/|W|
    above = np.nonzero(rel > tol)[0]
    for k in above[:20]:
        ratio = ref_abs[~zero][k] / abs(ref[~zero][k])
        print(f"  entry {k}: W {ref[~zero][k]:+.3e}, plain rel {rel[k]:.2e}, "
              f"sum|terms|/|W| {ratio:.2e}, rel/ratio {rel[k] / ratio:.2e}")
    assert err.max() <= tol, f"max scaled error {err.max():.3e}"
    return err.max()


def test_generator_device_equals_host():
    n, bc = (4, 6, 4, 8), 0
    host = generate_links(n, bc, 1234, 0.27)
    with Context(n, bc, "fp64") as c:
        c.generate(1234, 0.27)
        dev = c.download()
    assert np.array_equal(dev.view(np.uint64), host.view(np.uint64))


def test_upload_download_roundtrip():
    n = (4, 4, 6, 4)
    u = generate_links(n, 3, 5, 0.3)
    with Context(n, 3, "fp64") as c:
        c.upload(u)
        assert np.array_equal(c.download(), u)
    with Context(n, 3, "mixed") as c:
        c.upload(u)
        d = c.download()
        assert np.abs(d - u).max() < 1e-7


def _openqcd_ipt(n):
    """An openQCD-style ipt[]: even sites first, then odd (lexicographic within)."""
    x = np.indices(n).reshape(4, -1)
    par = x.sum(axis=0) % 2
    ipt = np.empty(x.shape[1], dtype=np.int32)
    ev = np.nonzero(par == 0)[0]
    od = np.nonzero(par == 1)[0]
    ipt[ev] = np.arange(len(ev))
    ipt[od] = len(ev) + np.arange(len(od))
    return ipt


def _to_openqcd(u, n, ipt):
    """Host-side packing into the openQCD layout (lnkcom.c:840-859)."""
    vol = int(np.prod(n))
    ud = np.zeros((4 * vol, 3, 3), dtype=np.complex128)
    U = L.as5d(u, n)
    inv = np.empty(vol, dtype=np.int64)
    inv[ipt] = np.arange(vol)
    xs = np.array(np.unravel_index(np.arange(vol), n)).T
    for iq in range(vol // 2, vol):
        s = inv[iq]
        x = xs[s]
        for mu in range(4):
            ud[8 * (iq - vol // 2) + 2 * mu] = U[tuple(x)][mu]
            y = x.copy()
            y[mu] = (y[mu] - 1) % n[mu]
            ud[8 * (iq - vol // 2) + 2 * mu + 1] = U[tuple(y)][mu]
    return ud


def test_openqcd_layout():
    n = (4, 4, 4, 6)
    u = generate_links(n, 3, 9, 0.3)
    ipt = _openqcd_ipt(n)
    ud = _to_openqcd(u, n, ipt)
    with Context(n, 3, "fp64") as c:
        c.upload_openqcd(ud, ipt)
        assert np.array_equal(c.download(), u)
        back = c.download_openqcd(ipt)
        assert np.array_equal(back, ud)


def test_projection():
    rng = np.random.default_rng(3)
    m = (rng.standard_normal((300, 3, 3)) + 1j * rng.standard_normal((300, 3, 3))) * 0.4 + np.eye(3)
    m[7] = 0.0
    ref = O.project(m, 6)
    got = np.ascontiguousarray(m.copy())
    approx_project_to_su3(got, 6)
    assert np.all(got[7] == 0.0)
    assert np.abs(got - ref).max() < 1e-14


def test_staple_sum():
    n = (4, 4, 2, 6)
    u1 = generate_links(n, 3, 1, 0.3)
    u2 = generate_links(n, 3, 2, 0.3)
    vb = generate_links(n, 3, 3, 0.3)
    for mu, nu in [(0, 2), (3, 1), (1, 0)]:
        ref = O.staple_sum(n, u1, u2, mu, nu, vb)
        got = vb.copy()
        staple_sum(n, u1, u2, mu, nu, got)
        assert np.abs(got - ref).max() < 1e-14


@pytest.mark.parametrize("bc", [0, 3])
def test_plaquette(bc):
    n = (6, 4, 4, 8)
    u = generate_links(n, bc, 17, 0.3)
    ref = O.plaq_sum(n, bc, u)
    for prec, tol in [("fp64", 1e-13), ("mixed", 1e-6)]:
        with Context(n, bc, prec) as c:
            c.upload(u)
            assert abs(c.lnk_plaq_sum() - ref) / abs(ref) < tol


@pytest.mark.parametrize("bc", [0, 3])
@pytest.mark.parametrize("mask", ["all", "time", "space"])
def test_hyp(bc, mask):
    n = (4, 6, 4, 4)
    u = generate_links(n, bc, 23, 0.3)
    t, s = {"all": (1, 1), "time": (1, 0), "space": (0, 1)}[mask]
    ref = O.hyp_links(n, bc, u, 1.0, 1.0, 0.5, 1, 4, time=t, space=s)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        {"all": c.hyp_links, "time": c.hyp_time_links, "space": c.hyp_space_links}[mask](
            1.0, 1.0, 0.5, 1, 4)
        got = c.download()
    assert np.abs(got - ref).max() < 1e-13


def test_hyp_no_projection_and_skip():
    n = (4, 4, 4, 4)
    u = generate_links(n, 3, 29, 0.3)
    ref = O.hyp_links(n, 3, u, 0.75, 0.6, 0.3, 0, 0)
    with Context(n, 3, "fp64") as c:
        c.upload(u)
        c.hyp_links(0.75, 0.6, 0.3, 0, 0)
        assert np.abs(c.download() - ref).max() < 1e-13
        c.upload(u)
        c.hyp_links(0.0, 0.6, 0.3, 1, 4)  # a1 == 0: no-op (hyp_links.c:405)
        assert np.array_equal(c.download(), u)


@pytest.mark.parametrize("time", [0, 1])
def test_ape(time):
    n = (4, 4, 6, 4)
    u = generate_links(n, 3, 31, 0.3)
    ref = O.ape_links(n, u, 0.5, 1, 4, time=time, nsweeps=3)
    with Context(n, 3, "fp64") as c:
        c.upload(u)
        (c.ape_links if time else c.ape_spatial_links)(0.5, 1, 4, nsweeps=3)
        got = c.download()
    assert np.abs(got - ref).max() < 1e-13


def test_hyp_spatial():
    n = (4, 4, 4, 6)
    u = generate_links(n, 3, 37, 0.3)
    ref = O.hyp_spatial_links(n, u, 0.75, 0.3, 1, 4, nsweeps=2)
    with Context(n, 3, "fp64") as c:
        c.upload(u)
        c.hyp_spatial_links(0.75, 0.3, 1, 4, nsweeps=2)
        got = c.download()
    assert np.abs(got - ref).max() < 1e-13


CASES = [
    # (n, bc, parms)
    ((8, 8, 8, 8), 3, WloopParms(msl=4, nss=[0, 5, 5, 5], mwlt=4, mwlr=4, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),                 # the 8^4 workload
    ((8, 4, 6, 4), 0, WloopParms(msl=3, nss=[0, 2, 2], mwlt=5, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((6, 4, 4, 4), 3, WloopParms(msl=3, nss=[0, 1, 2], mwlt=4, mwlr=3, op_smear=HYP,
                                 alpha_hyp=(0.75, 0.3), proj_iter=4)),
    ((4, 4, 4, 4), 0, WloopParms(msl=5, nss=[0, 1, 0, 1, 1], mwlt=3, mwlr=3, op_smear=APE,
                                 alpha_ape=0.4, proj_iter=0)),
    ((10, 6, 6, 6), 0, WloopParms(msl=6, nss=[0, 2, 2, 2, 2, 2], mwlt=6, mwlr=4, op_smear=APE,
                                  alpha_ape=0.5, proj_iter=4)),
    # level counts at the ends of the range (1, 2, 7 and MAX_SM_LEVELS = 8) and
    # odd extents (time slices of 105 sites, not a multiple of the 32-site tile)
    ((6, 4, 4, 4), 3, WloopParms(msl=1, nss=[3], mwlt=4, mwlr=3, op_smear=APE, alpha_ape=0.5,
                                 proj_iter=4)),
    ((7, 5, 3, 7), 3, WloopParms(msl=2, nss=[0, 2], mwlt=4, mwlr=2, op_smear=APE, alpha_ape=0.5,
                                 proj_iter=4)),
    ((6, 4, 6, 4), 0, WloopParms(msl=7, nss=[0, 1, 1, 1, 1, 1, 1], mwlt=4, mwlr=3, op_smear=APE,
                                 alpha_ape=0.5, proj_iter=4)),
    ((4, 4, 4, 6), 3, WloopParms(msl=8, nss=[1, 1, 0, 1, 1, 1, 0, 1], mwlt=3, mwlr=3,
                                 op_smear=HYP, alpha_hyp=(0.6, 0.3), proj_iter=3)),
    # the largest loops the parameters allow (mwlt = N0/2+1, mwlr = min Nk/2+1,
    # wloop_parms.c:174-176): temporal and spatial lines wrap around the
    # periodic lattice, and with open bc every loop longer than the remaining
    # time extent vanishes
    ((8, 4, 6, 4), 3, WloopParms(msl=2, nss=[0, 3], mwlt=5, mwlr=3, op_smear=APE, alpha_ape=0.5,
                                 proj_iter=4)),
    ((8, 4, 6, 4), 0, WloopParms(msl=2, nss=[2, 1], mwlt=5, mwlr=3, op_smear=APE, alpha_ape=0.45,
                                 proj_iter=4)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_wloop_sum_fp64(case):
    n, bc, p = CASES[case]
    u = generate_links(n, bc, 100 + case, 0.25)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref, ref_abs, ref_plaq = O.wloop_sum(n, bc, uh, p, want_abs=True, want_plaq=True)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        got, plaq = c.measure(p, plaq=True)
    assert_wl_close(got, ref, ref_abs)
    assert np.abs(plaq - ref_plaq).max() / np.abs(ref_plaq).max() < 1e-12


@pytest.mark.parametrize("case", [0, 1, 3, 4, 6, 8, 9, 10])
def test_wloop_sum_mixed(case):
    n, bc, p = CASES[case]
    u = generate_links(n, bc, 100 + case, 0.25)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref, ref_abs = O.wloop_sum(n, bc, uh, p, want_abs=True)
    with Context(n, bc, "mixed") as c:
        c.upload(u)
        got = c.measure(p)
    zero = ref == 0.0
    assert np.all(got[zero] == 0.0)
    rel = np.abs(got - ref)[~zero] / np.abs(ref)[~zero]
    scaled = np.abs(got - ref)[~zero] / np.maximum(np.abs(ref), ref_abs)[~zero]
    print(f"mixed vs oracle: max rel {rel.max():.2e}, max scaled {scaled.max():.2e}")
    # the mixed form's bar: every non-zero entry within 1e-6 plain relative
    # of the FP64 oracle
    assert rel.max() <= 1e-6, f"max plain relative error {rel.max():.3e}"


@pytest.mark.parametrize("bc", [0, 3])
def test_unit_field(bc):
    """devel/wloop/check1.c on the GPU (W = 1, crossing loops 0)."""
    n = (8, 4, 4, 4)
    p = WloopParms(msl=4, nss=[0, 1, 2, 3], mwlt=4, mwlr=3, op_smear=APE, alpha_ape=0.5,
                   proj_iter=10)
    u = L.unit_field(n, bc)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        c.hyp_time_links(1.0, 1.0, 0.5, 1, 10)
        wl = c.wloop_sum(p).reshape(n[0], p.mwlr, p.mwlt, p.msl, p.msl)
    eps = np.sqrt(3.0) * n[0] * n[1] / 4 * np.finfo(float).eps
    for x0 in range(n[0]):
        for t in range(p.mwlt):
            if bc == 0 and x0 + t + 1 > n[0] - 1:
                assert np.all(wl[x0, :, t] == 0.0)
            else:
                assert np.abs(wl[x0, :, t] - 1.0).max() < eps


def test_gauge_invariance_gpu():
    """devel/wloop/check2.c on the GPU at 8^3x16, open bc."""
    n, bc = (16, 8, 8, 8), 0
    p = WloopParms(msl=3, nss=[0, 2, 3], mwlt=6, mwlr=4, op_smear=HYP, alpha_hyp=(1.0, 0.5),
                   proj_iter=0)
    u = generate_links(n, bc, 77, 0.3)
    g = L.random_su3(tuple(n), np.random.default_rng(5))
    ug = L.gauge_transform(u, n, bc, g)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        w1 = c.measure(p)
        c.upload(ug)
        w2 = c.measure(p)
    eps = 100 * np.sqrt(p.msl ** 2 * p.mwlr * p.mwlt * 3 * np.prod(n)) * np.finfo(float).eps
    nz = w1 != 0
    assert np.array_equal(w2 == 0, ~nz)
    assert np.abs(1.0 - w2[nz] / w1[nz]).max() < eps


def test_levels_match_oracle():
    n, bc = (6, 4, 4, 4), 3
    p = WloopParms(msl=3, nss=[1, 2, 0], mwlt=2, mwlr=2, op_smear=APE, alpha_ape=0.5, proj_iter=4)
    u = generate_links(n, bc, 3, 0.3)
    _, lv = O.wloop_sum(n, bc, u, p, want_levels=True)
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        c.wloop_sum(p)
        for sl in range(p.msl):
            assert np.abs(c.level(sl) - lv[sl]).max() < 1e-13


def test_parameter_errors():
    n = (4, 4, 4, 4)
    with Context(n, 3, "fp64") as c:
        for p in [WloopParms(msl=9, nss=[0] * 8, mwlt=1, mwlr=1),
                  WloopParms(msl=1, nss=[0], mwlt=4, mwlr=1),
                  WloopParms(msl=1, nss=[0], mwlt=1, mwlr=4),
                  WloopParms(msl=1, nss=[0], mwlt=1, mwlr=1, op_smear=5)]:
            with pytest.raises(Exception):
                c.wloop_sum(p)


# every contraction form and shape the tuner or a caller may pick gives the
# default's result up to summation order (including 32-thread blocks with an
# odd number of per-warp row doubles, where the line stage must still start on
# a 16-byte boundary)
SHAPES = [  # (form, G, SB, nCB, block)
    (2, 1, 1, 0, 64), (2, 3, 2, 0, 128), (3, 1, 2, 0, 64), (3, 3, 1, 0, 128), (3, 2, 2, 5, 96),
    (4, 3, 0, 0, 32), (4, 1, 0, 7, 64), (4, 2, 0, 0, 128), (5, 3, 0, 0, 32), (5, 2, 0, 3, 64),
    (5, 4, 0, 0, 128),
    # bulk-copy staging (forms 6 and 7; on lattices whose time slices are not
    # whole 32-site tiles they run as forms 5 and 4)
    (6, 3, 0, 0, 128), (6, 2, 0, 5, 32), (7, 3, 0, 0, 64), (7, 1, 0, 0, 96), (6, 4, 0, 3, 64),
    # packed FP32 products (form 8; an FP64 context runs form 5)
    (8, 3, 0, 0, 128), (8, 2, 0, 3, 64), (8, 4, 0, 0, 32), (8, 1, 0, 0, 96),
]


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("case", [0, 1, 4, 8])
def test_contract_shapes(case, prec):
    n, bc, p = CASES[case]
    u = generate_links(n, bc, 300 + case, 0.25)
    with Context(n, bc, prec) as c:
        c.set_contract_tuning(variant=carried_form(prec))
        c.upload(u)
        c.snapshot()
        ref = c.measure(p)
        scale = np.maximum(np.abs(ref), 1e-3)
        for form, G, SB, ncb, block in SHAPES:
            if G > p.msl:
                continue
            c.set_contract_tuning(form, G, SB, ncb, block)
            c.restore()
            got = c.measure(p)
            tol = 1e-13 if prec == "fp64" else 1e-6
            assert np.max(np.abs(got - ref) / scale) < tol, (form, G, SB, ncb, block)


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_prefetched_upload(prec):
    """The pipelined upload (copy on the copy stream, transposition on the
    context's stream) gives the field an ordinary upload gives, also while a
    measurement is running, and refuses misuse."""
    n, bc, p = CASES[1]
    u1 = generate_links(n, bc, 41, 0.25)
    u2 = generate_links(n, bc, 42, 0.25)
    with Context(n, bc, prec) as c:
        c.upload(u2)
        ref2 = c.measure(p)
        c.upload(u1)
        ref1 = c.measure(p)
        with pytest.raises(Exception, match="no field was prefetched"):
            c.upload_prefetched()
        c.prefetch(u2)
        with pytest.raises(Exception, match="has not been uploaded"):
            c.prefetch(u1)
        c.upload_prefetched()
        c.prefetch(u1)          # overlaps the next measurement
        assert np.array_equal(c.measure(p), ref2)
        c.upload_prefetched()
        assert np.array_equal(c.measure(p), ref1)


@pytest.mark.parametrize("prec,form", [("fp64", 0), ("fp64", 3), ("fp64", 11), ("mixed", 0),
                                       ("mixed", 3), ("mixed", 11)])
def test_lines_left_by_the_measurement(prec, form):
    """The spatial lines a measurement leaves (get_pus slots msl..2msl-1) are
    the products of mwlr level links along each direction, whether the
    contraction computed them (fourth-form family) or the line-step stage did
    (third form), or they are rebuilt from the level store after a
    temporal-gauge measurement (form 11)."""
    n, bc, p = CASES[1]
    u = generate_links(n, bc, 77, 0.25)
    with Context(n, bc, prec) as c:
        if form:
            c.set_contract_tuning(form, 2, 1, 0, 64)
        c.upload(u)
        c.measure(p)
        st = np.array([n[1] * n[2] * n[3], n[2] * n[3], n[3], 1])
        x = np.indices(n).reshape(4, -1).T
        for sl in range(p.msl):
            lev = c.level(sl)
            got, length = c.lines(sl)
            assert length == p.mwlr
            for k in range(3):
                want = lev[:, k].copy()
                for step in range(1, length):
                    y = x.copy()
                    y[:, k + 1] = (y[:, k + 1] + step) % n[k + 1]
                    want = want @ lev[y @ st, k]
                tol = 1e-13 if prec == "fp64" else 2e-6
                assert np.max(np.abs(got[:, k] - want)) < tol, (sl, k)


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 3, 4])
def test_ninth_form_matches_default(case):
    """The ninth contraction form (one 32-column chunk per warp, per-warp
    partial records) gives the tenth form's mixed result up to the order of
    the FP64 sums, and the oracle's within 1e-6 plain relative."""
    n, bc, p = CASES[case]
    u = generate_links(n, bc, 700 + case, 0.25)
    uh = O.hyp_links(n, bc, u, *p.alpha_action, p.proj, p.proj_iter)
    ref = O.wloop_sum(n, bc, uh, p)
    with Context(n, bc, "mixed") as c:
        c.set_contract_tuning(variant=10)
        c.upload(u)
        base = c.measure(p)
        c.set_contract_tuning(variant=9)
        c.upload(u)
        got = c.measure(p)
    nz = ref != 0.0
    assert np.all(got[~nz] == 0.0)
    assert np.abs(got - base).max() <= 1e-13 * np.abs(base).max()
    assert (np.abs(got - ref)[nz] / np.abs(ref)[nz]).max() <= 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 4])
def test_tenth_form_is_the_eighth_bit_for_bit(case):
    """Form 10 moves the signs of the packed products into the shared
    broadcast pairs: the same products, so the same result as form 8."""
    n, bc, p = CASES[case]
    u = generate_links(n, bc, 710 + case, 0.25)
    out = []
    for v in (8, 10):
        with Context(n, bc, "mixed") as c:
            c.set_contract_tuning(variant=v)
            c.upload(u)
            out.append(c.measure(p))
    assert np.array_equal(out[0], out[1])
