"""Serving loop (wlg_server): continuous batching of measurement requests.

The result of a request is identical alone and in a mix of concurrent
requests of other lattices (same per-lattice arithmetic and reduction order
in every batch), and identical to a context's wlg_measure on the same field;
requests that cannot fit the memory budget fail with a message instead of
blocking the queue.
"""
import time

import numpy as np
import pytest

from wloop_b200 import APE, Context, WloopParms, generate_links
from wloop_b200.api import Server, estimate_bytes

P = WloopParms(msl=3, nss=[0, 2, 2], mwlt=3, mwlr=2, op_smear=APE, alpha_ape=0.5, proj_iter=4)


def test_estimate_bytes_scales_with_volume():
    a = estimate_bytes((8, 4, 4, 4), 3, P, "mixed")
    b = estimate_bytes((16, 8, 8, 8), 3, P, "mixed")
    c = estimate_bytes((16, 8, 8, 8), 3, P, "fp64")
    assert 0 < a < b < c
    assert b > 8 * a


@pytest.mark.gpu
def test_result_same_alone_and_in_mix():
    x = ((8, 4, 4, 4), 3, 4711, 0.25)
    with Server(max_inflight=2, max_batch=4) as s:
        rid = s.submit(x[0], x[1], P, "mixed", seed=x[2], eps=x[3])
        alone, lat, bs = s.wait(rid)
        assert bs == 1 and lat > 0
    others = [((6, 4, 6, 4), 0, 11, 0.3), ((8, 4, 4, 4), 0, 12, 0.2), ((8, 4, 4, 4), 3, 13, 0.3),
              ((12, 6, 6, 6), 3, 14, 0.2), ((8, 4, 4, 4), 3, 15, 0.35)]
    with Server(max_inflight=3, max_batch=4) as s:
        ids = []
        for k, o in enumerate(others):
            ids.append(s.submit(o[0], o[1], P, "mixed", seed=o[2], eps=o[3]))
            if k == 1:
                mine = s.submit(x[0], x[1], P, "mixed", seed=x[2], eps=x[3])
        mixed_res, _, bs_mix = s.wait(mine)
        outs = [s.wait(i) for i in ids]
        st = s.stats()
    assert np.array_equal(alone, mixed_res), "result differs alone vs in the mix"
    assert st["completed"] == len(others) + 1 and st["failed"] == 0
    assert st["p99_ms"] >= st["p50_ms"] > 0
    # every result equals a plain context measurement of the same field
    for o, (res, _, _) in zip(others, outs):
        with Context(o[0], o[1], "mixed") as c:
            c.generate(o[2], o[3])
            assert np.array_equal(c.measure(P), res)


@pytest.mark.gpu
def test_host_field_request_matches_context():
    n, bc = (8, 6, 4, 4), 0
    u = generate_links(n, bc, 99, 0.3)
    with Server(max_inflight=1) as s:
        res, _, _ = s.wait(s.submit(n, bc, P, "fp64", links=u))
    with Context(n, bc, "fp64") as c:
        c.upload(u)
        assert np.array_equal(c.measure(P), res)


@pytest.mark.gpu
def test_request_over_budget_fails_cleanly():
    with Server(mem_fraction=1e-6, max_inflight=1) as s:
        rid = s.submit((8, 4, 4, 4), 3, P, "mixed", seed=1)
        with pytest.raises(Exception, match="budget"):
            s.wait(rid)
        assert s.stats()["failed"] == 1


@pytest.mark.gpu
def test_requests_overlap_and_batch():
    with Server(max_inflight=2, max_batch=8) as s:
        t0 = time.time()
        ids = [s.submit((8, 4, 4, 4), 3, P, "mixed", seed=100 + i, eps=0.2) for i in range(12)]
        res = [s.wait(i) for i in ids]
        st = s.stats()
    assert st["completed"] == 12
    assert st["batches"] < 12  # requests that queued together were measured together
    assert max(bs for _, _, bs in res) > 1


@pytest.mark.gpu
def test_budget_counts_memory_the_batch_pool_keeps():
    """Batches return their memory to a pool that keeps it for the next
    batch; a server created afterwards counts that idle memory as free, and
    a context allocation gets it back from the pool when the device is full."""
    from wloop_b200._native import lib
    from wloop_b200.api import Batch
    items = [((16, 8, 8, 8), 3, P)] * 4
    with Batch(items, "mixed") as b:
        b.generate([1, 2, 3, 4], [0.2] * 4)
        b.run()
        held = b.device_bytes
    idle = lib.wlg_batch_pool_idle_bytes(0)
    assert idle >= held
    with Server(mem_fraction=0.5) as s:
        assert s.budget >= 0.5 * idle


# a request that takes the GPU about a tenth of a second
BIG_N = (64, 32, 32, 32)
BIG_P = WloopParms(msl=4, nss=[0, 10, 10, 10], mwlt=16, mwlr=12, op_smear=APE, alpha_ape=0.5,
                   proj_iter=4)


def _bypass_run(bypass_ms):
    """A large request A runs; a second large request B waits at the head of
    the queue (the budget holds one large and two small requests); small
    requests C, D behind B.  Returns the completion times of A and C."""
    small = (8, 4, 4, 4)
    with Server(max_inflight=3, max_batch=1) as s:
        s.set_limits(budget_bytes=estimate_bytes(BIG_N, 3, BIG_P, "fp64") +
                     2 * estimate_bytes(small, 3, P, "fp64") + 1024, bypass_ms=bypass_ms)
        done = {}
        t0 = time.perf_counter()
        ids = {k: (s.submit(n, 3, p, "fp64", seed=k + 1, eps=0.25), time.perf_counter())
               for k, (n, p) in enumerate([(BIG_N, BIG_P), (BIG_N, BIG_P), (small, P),
                                           (small, P)])}
        for k, (rid, ts) in ids.items():
            _, lat, _ = s.wait(rid)
            done[k] = ts - t0 + lat * 1e-3
        assert s.stats()["failed"] == 0
    return done[0], done[2]


@pytest.mark.gpu
def test_head_of_line_request_is_bypassed_then_protected():
    """A small request that fits starts before an older large one that does
    not fit yet; with a zero bypass limit it waits behind it instead."""
    a_done, c_done = _bypass_run(bypass_ms=60000.0)
    assert c_done < a_done  # C ran beside A, before B
    a_done, c_done = _bypass_run(bypass_ms=0.0)
    assert c_done > a_done  # C waited for B, which waited for A


@pytest.mark.gpu
def test_mixed_lattices_share_a_batch_and_match_alone():
    """Requests of different lattices and level counts in one batch give what
    each gives alone."""
    q = WloopParms(msl=2, nss=[1, 2], mwlt=2, mwlr=2, op_smear=APE, alpha_ape=0.5, proj_iter=4)
    reqs = [((8, 4, 4, 4), 3, P, 21), ((6, 4, 6, 4), 0, q, 22), ((12, 6, 6, 6), 3, P, 23)]
    with Server(max_inflight=1, max_batch=8) as s:
        # the one worker is busy with a large request while the three queue
        blocker = s.submit(BIG_N, 3, BIG_P, "mixed", seed=20, eps=0.3)
        ids = [s.submit(n, bc, p, "mixed", seed=sd, eps=0.3) for n, bc, p, sd in reqs]
        s.wait(blocker)
        outs = [s.wait(i) for i in ids]
    assert max(bs for _, _, bs in outs) > 1
    for (n, bc, p, sd), (res, _, _) in zip(reqs, outs):
        with Context(n, bc, "mixed") as c:
            c.generate(sd, 0.3)
            assert np.array_equal(c.measure(p), res)
