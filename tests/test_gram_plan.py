"""The temporal-gauge form's launch plan, checked on the CPU (no GPU: the SM
count defaults to 148) over many lattices, level counts, time extents and
tunings: the invariants the Gram kernel's indexing relies on (block and
shared-memory limits, the staged rows a thread reads, the swizzle's 8-row
alignment, full coverage of the start slices and the column chunks, 32-bit
row offsets) and the FP32 column-run cap."""
import ctypes as C
import itertools
import math

import pytest

from wloop_b200._native import WLG_FP64, WLG_MIXED, lib

KEYS = ("tq", "occ", "ord", "bx", "bxp", "ng", "nyb", "nybp", "nblk", "nrows", "stages", "block",
        "smem", "nchunks", "cpc", "nsplit")


def plan(n, bc, msl, mwlt, prec, tune=None):
    nn = (C.c_int * 4)(*n)
    t = (C.c_int * 5)(*(tune or (0, 0, 0, 0, 0)))
    out = (C.c_longlong * 16)()
    rc = lib.wlg_gram_plan_shape(nn, bc, msl, mwlt, prec, t, out)
    return dict(zip(KEYS, list(out))) if rc == 0 else None


LATTICES = [(4, 4, 4, 4), (8, 4, 6, 4), (7, 5, 3, 7), (10, 6, 6, 6), (40, 4, 4, 4), (8, 16, 16, 16),
            (32, 16, 16, 16), (48, 24, 24, 24), (64, 32, 32, 32), (96, 48, 48, 48)]


def check(n, bc, msl, mwlt, prec, p, tune=None):
    N0 = n[0]
    vs = n[1] * n[2] * n[3]
    esz = 8 if prec == WLG_FP64 else 4
    threads = {1: 256, 2: 192, 3: 384}[p["occ"]]
    assert p["block"] % 32 == 0 and p["bx"] * p["ng"] <= p["block"] <= threads
    assert p["ng"] * p["tq"] >= mwlt and (p["ng"] - 1) * p["tq"] < mwlt
    assert p["nblk"] * p["bx"] >= N0 > (p["nblk"] - 1) * p["bx"]
    assert p["bxp"] % 8 == 0 and p["bxp"] - 8 < p["bx"] <= p["bxp"]
    assert p["nyb"] == p["bx"] + mwlt - 1
    assert p["nybp"] % 8 == 0 and p["nybp"] - 8 < p["nyb"] <= p["nybp"]
    assert p["nrows"] == msl * (p["bxp"] + p["nybp"])
    # the largest row a thread reads: its last B row of the last level
    assert (msl - 1) * p["nybp"] + p["bx"] - 1 + mwlt - 1 < msl * p["nybp"]
    tab = (p["nrows"] * 4 + 127) & ~127
    assert p["stages"] >= 2 and p["smem"] == tab + p["stages"] * p["nrows"] * 128
    assert p["smem"] <= (113 if p["occ"] == 2 else 227) * 1024
    ntile = (vs + 31) // 32
    assert p["nchunks"] == 3 * ntile * 18 * (32 * esz // 128)
    assert p["nsplit"] * p["cpc"] >= p["nchunks"] > (p["nsplit"] - 1) * p["cpc"]
    nu = N0 + (0 if bc == 0 else mwlt)
    assert 3 * msl * nu * ntile * 576 * esz // 16 < 2 ** 32 - 1
    if prec == WLG_MIXED and not (tune and tune[4]):
        assert p["cpc"] <= max(1, int(2 * math.sqrt(p["nchunks"] / 32)))


@pytest.mark.parametrize("prec", [WLG_FP64, WLG_MIXED])
@pytest.mark.parametrize("n", LATTICES)
def test_default_plans(n, prec):
    for bc, msl in itertools.product((0, 3), (1, 2, 3, 4, 5, 6, 7, 8)):
        for mwlt in sorted({1, 2, 3, n[0] // 4 + 1, n[0] // 2 + 1}):
            p = plan(n, bc, msl, mwlt, prec)
            assert p is not None, (n, bc, msl, mwlt)
            check(n, bc, msl, mwlt, prec, p)


@pytest.mark.parametrize("prec", [WLG_FP64, WLG_MIXED])
def test_tuned_plans(prec):
    n, bc, msl, mwlt = (64, 32, 32, 32), 3, 6, 24
    for occ, ord_, bx, stages, cpc in itertools.product((0, 1, 2, 3), (0, 1, 2), (0, 8, 22, 32),
                                                        (0, 2, 3), (0, 24, 96)):
        tune = (occ, ord_, bx, stages, cpc)
        p = plan(n, bc, msl, mwlt, prec, tune)
        if p is None:
            continue  # no kernel of that occupancy for this precision and msl
        check(n, bc, msl, mwlt, prec, p, tune)
        if occ:
            assert p["occ"] == occ
        if bx:
            assert p["bx"] <= bx
        if cpc:
            assert p["cpc"] == cpc


def test_c3_default_shapes():
    """The 32^3x64 plans the measurements in the profiles ran."""
    p = plan((64, 32, 32, 32), 3, 6, 24, WLG_MIXED)
    assert (p["occ"], p["tq"], p["bx"], p["nblk"], p["stages"], p["cpc"], p["nsplit"]) == \
        (1, 3, 32, 2, 3, 75, 738)
    p = plan((64, 32, 32, 32), 3, 6, 24, WLG_FP64)
    assert (p["occ"], p["tq"], p["bx"], p["nblk"], p["cpc"], p["nsplit"]) == (2, 1, 8, 8, 499, 222)


def test_plans_refused():
    """Level counts outside 1..8, a time extent whose extent groups exceed a
    block, or an unknown precision give -1 and a message, not a plan."""
    n = (64, 32, 32, 32)
    for msl, mwlt, prec in ((0, 4, WLG_MIXED), (9, 4, WLG_FP64), (6, 0, WLG_MIXED),
                            (6, 4000, WLG_MIXED), (6, 4000, WLG_FP64), (6, 4, 7)):
        assert plan(n, 3, msl, mwlt, prec) is None, (msl, mwlt, prec)
        assert lib.wlg_last_error()
    assert plan(n, 3, 6, 24, WLG_MIXED) is not None
    # lattices and boundary conditions a context refuses
    for bad, bc in (((0, 4, 4, 4), 3), ((8, 1, 4, 4), 3), ((-8, 4, 4, 4), 0),
                    ((2048, 1024, 1024, 2), 3), ((8, 4, 4, 4), 1)):
        assert plan(bad, bc, 2, 2, WLG_MIXED) is None, bad
        assert lib.wlg_last_error()


def test_batch_estimate_refuses_bad_lattices():
    """The batch memory estimate (host only, used by the serving loop's
    admission) refuses what wlg_batch_create refuses, instead of planning a
    lattice with a zero extent."""
    from wloop_b200 import APE, WloopParms
    from wloop_b200.api import estimate_bytes
    p = WloopParms(msl=2, nss=[0, 1], mwlt=1, mwlr=1, op_smear=APE, alpha_ape=0.5, proj_iter=4)
    assert estimate_bytes((8, 4, 4, 4), 3, p, "mixed") > 0
    assert estimate_bytes((64, 32, 32, 32), 3, p, "fp64") > estimate_bytes((64, 32, 32, 32), 3, p)
    for n, bc in (((0, 4, 4, 4), 3), ((8, 0, 4, 4), 3), ((8, 4, 4, 4), 1),
                  ((2048, 1024, 1024, 2), 3)):
        assert estimate_bytes(n, bc, p, "mixed") == -1, (n, bc)
