"""Measurement runs and their output files.

CPU: the .dat and .par byte layouts of main/ms10.c:86-190 and
wloop_parms.c:343-382 (written through the library, read back with numpy),
torn-record and head checks, and the replica path over two gloo ranks: the
rank-sharded files merged give byte for byte the file one process writes,
the maximum over ranks is the slowest rank's, and a rank that leaves makes
the other's next collective fail instead of hang.
GPU: a run measures every configuration as a context does alone, and its FP64
records match the oracle.
"""
import os
import socket
import struct
import time

import numpy as np
import pytest

from wloop_b200 import APE, HYP, WloopParms
from wloop_b200._native import WlgError
from wloop_b200 import measure as M
from wloop_b200.replicas import config_numbers, shard

P = WloopParms(msl=3, nss=[0, 1, 2], mwlt=3, mwlr=2, op_smear=APE, alpha_ape=0.5, proj_iter=4)
N = (8, 4, 4, 4)


def fake_wl(nc: int, wls: int) -> np.ndarray:
    rng = np.random.default_rng(nc)
    return rng.standard_normal(wls)


def test_dat_layout(tmp_path):
    head = M.dat_head(P, N[0])
    assert head == [3 * 3 * 3 * 2 * 8, 3, 3, 2, 8]
    path = str(tmp_path / "a.dat")
    M.write_head(path, head)
    recs = {7: fake_wl(7, head[0]), 9: fake_wl(9, head[0]), 11: fake_wl(11, head[0])}
    for nc, wl in recs.items():
        M.append(path, nc, wl)
    raw = open(path, "rb").read()
    assert len(raw) == 20 + 3 * (4 + 8 * head[0])
    assert list(struct.unpack("<5i", raw[:20])) == head
    off = 20
    for nc, wl in recs.items():
        assert struct.unpack("<i", raw[off:off + 4])[0] == nc
        got = np.frombuffer(raw[off + 4:off + 4 + 8 * head[0]], dtype="<f8")
        assert np.array_equal(got, wl)
        off += 4 + 8 * head[0]
    h, ncs, wl = M.read(path)
    assert h == head and list(ncs) == [7, 9, 11]
    assert np.array_equal(wl[1], recs[9])
    M.check_head(path, head)
    with pytest.raises(WlgError, match="Unexpected value"):
        M.check_head(path, [head[0], 3, 3, 2, 9])


def test_dat_torn_record_and_bad_head(tmp_path):
    head = M.dat_head(P, N[0])
    path = str(tmp_path / "t.dat")
    M.write_head(path, head)
    M.append(path, 1, fake_wl(1, head[0]))
    with open(path, "ab") as f:  # a record cut short, as by a killed writer
        f.write(b"\x02\x00\x00\x00" + b"\x00" * 16)
    with pytest.raises(WlgError, match="incomplete data record"):
        M.count(path)
    with pytest.raises(WlgError, match="wls"):
        M.write_head(str(tmp_path / "b.dat"), [head[0] + 1] + head[1:])
    with pytest.raises(WlgError):
        M.append(path, 3, np.zeros(0))


def test_par_layout(tmp_path):
    path = str(tmp_path / "r.par")
    p = WloopParms(msl=2, nss=[3, 4], mwlt=5, mwlr=6, op_smear=HYP, alpha_action=(0.75, 0.6, 0.3),
                   alpha_ape=0.0, alpha_hyp=(0.7, 0.2), proj_iter=3)
    M.write_par(path, p)
    raw = open(path, "rb").read()
    assert len(raw) == 4 * (2 + 4) + 8 * 6
    assert struct.unpack("<6i", raw[:24]) == (3, 4, 5, 6, HYP, 3)
    assert struct.unpack("<6d", raw[24:]) == (0.0, 0.7, 0.2, 0.75, 0.6, 0.3)
    M.check_par(path, p)
    q = WloopParms(msl=2, nss=[3, 4], mwlt=5, mwlr=6, op_smear=HYP, alpha_action=(0.75, 0.6, 0.3),
                   alpha_ape=0.0, alpha_hyp=(0.7, 0.25), proj_iter=3)
    with pytest.raises(WlgError, match="do not match"):
        M.check_par(path, q)


def test_par_bc_record_precedes_wloop_record(tmp_path):
    """The .par file as ms10 writes it (ms10.c:290-313): the boundary-condition
    record (int32 type, 10 doubles cG, cG', cF, cF', phi[3], phi'[3]) and then
    the wloop record."""
    for bc in (0, 3):
        path = str(tmp_path / f"bc{bc}.par")
        M.write_par(path, P, bc)
        raw = open(path, "rb").read()
        assert len(raw) == M.BC_RECORD_BYTES + 4 * (P.msl + 4) + 8 * 6
        assert struct.unpack("<i", raw[:4]) == (bc,)
        assert struct.unpack("<10d", raw[4:84]) == (1.0, 1.0, 1.0, 1.0) + (0.0,) * 6
        assert struct.unpack(f"<{P.msl}i", raw[84:84 + 4 * P.msl]) == tuple(P.nss[:P.msl])
        M.check_par(path, P, bc=bc)
        with pytest.raises(WlgError, match="do not match"):
            M.check_par(path, P, bc=3 - bc)
    with pytest.raises(WlgError, match="open"):
        M.write_par(str(tmp_path / "x.par"), P, 1)


def test_shard_covers_every_config_once():
    cfgs = config_numbers(3, 40, 4)
    assert cfgs[0] == 3 and cfgs[-1] <= 40 and len(cfgs) == 10
    for world in (1, 2, 3, 4, 8):
        parts = [shard(cfgs, r, world) for r in range(world)]
        flat = sorted(x for p in parts for x in p)
        assert flat == cfgs
        sizes = [len(p) for p in parts]
        assert max(sizes) - min(sizes) <= 1


def test_run_single_process_with_fake_measure(tmp_path):
    head = M.dat_head(P, N[0])
    r = M.Run("one", N, 3, P, first=2, last=10, step=2)
    res = M.run(r, str(tmp_path), measure=lambda nc: fake_wl(nc, head[0]))
    assert res["configs"] == [2, 4, 6, 8, 10]
    h, ncs, wl = M.read(str(tmp_path / "one.ms10.dat"))
    assert list(ncs) == [2, 4, 6, 8, 10]
    assert np.array_equal(wl[3], fake_wl(8, head[0]))
    M.check_par(str(tmp_path / "one.ms10.par"), P, bc=3)


# ---------------------------------------------------------------------------
# ms10's file safety, continuation (-a), end flag and backups
# ---------------------------------------------------------------------------
def _fake(head):
    return lambda nc: fake_wl(nc, head[0])


def test_new_run_refuses_to_overwrite(tmp_path):
    head = M.dat_head(P, N[0])
    M.run(M.Run("o", N, 3, P, first=1, last=3), str(tmp_path), measure=_fake(head))
    with pytest.raises(WlgError, match="overwrite"):
        M.run(M.Run("o", N, 3, P, first=1, last=3), str(tmp_path), measure=_fake(head))


def test_continuation_run_equals_one_run(tmp_path):
    head = M.dat_head(P, N[0])
    M.run(M.Run("c", N, 3, P, first=1, last=5, step=2), str(tmp_path / "a"), measure=_fake(head))
    res = M.run(M.Run("c", N, 3, P, first=7, last=11, step=2), str(tmp_path / "a"),
                measure=_fake(head), continue_run=True)
    assert res["configs"] == [7, 9, 11]
    M.run(M.Run("c", N, 3, P, first=1, last=11, step=2), str(tmp_path / "b"), measure=_fake(head))
    a = open(M.dat_path(str(tmp_path / "a"), "c"), "rb").read()
    b = open(M.dat_path(str(tmp_path / "b"), "c"), "rb").read()
    assert a == b
    log = open(M.log_path(str(tmp_path / "a"), "c")).read()
    assert log.count("fully processed") == 6
    # the backups follow the files
    for f in (M.dat_path(str(tmp_path / "a"), "c"), M.log_path(str(tmp_path / "a"), "c")):
        assert open(f, "rb").read() == open(f + "~", "rb").read()


@pytest.mark.parametrize("first,step,parms,match", [
    (9, 2, P, "does not continue"),
    (7, 3, P, "different configuration separation"),
    (7, 2, WloopParms(msl=3, nss=[0, 1, 3], mwlt=3, mwlr=2, op_smear=APE, alpha_ape=0.5,
                      proj_iter=4), "do not match"),
])
def test_continuation_checks(tmp_path, first, step, parms, match):
    head = M.dat_head(P, N[0])
    M.run(M.Run("k", N, 3, P, first=1, last=5, step=2), str(tmp_path), measure=_fake(head))
    with pytest.raises(WlgError, match=match):
        M.run(M.Run("k", N, 3, parms, first=first, last=first + 4, step=step), str(tmp_path),
              measure=_fake(head), continue_run=True)


def test_continuation_refuses_an_inconsistent_log(tmp_path):
    head = M.dat_head(P, N[0])
    M.run(M.Run("g", N, 3, P, first=1, last=5, step=2), str(tmp_path), measure=_fake(head))
    with open(M.log_path(str(tmp_path), "g"), "a") as f:
        f.write("Configuration no 7 fully processed in 1.00e+00 sec\n")
    with pytest.raises(WlgError, match="not as reported in the log"):
        M.run(M.Run("g", N, 3, P, first=9, last=9), str(tmp_path), measure=_fake(head),
              continue_run=True)


def test_end_flag_stops_the_run(tmp_path):
    head = M.dat_head(P, N[0])
    open(M.end_path(str(tmp_path), "e"), "w").close()
    res = M.run(M.Run("e", N, 3, P, first=1, last=9), str(tmp_path), measure=_fake(head))
    assert res["configs"] == [1]
    assert not os.path.exists(M.end_path(str(tmp_path), "e"))
    assert M.count(M.dat_path(str(tmp_path), "e"))[1] == 1
    assert "End flag set, run stopped" in open(M.log_path(str(tmp_path), "e")).read()


# ---------------------------------------------------------------------------
# two replicas over gloo
# ---------------------------------------------------------------------------
def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _replica_main(rank, world, port, out_dir, mode, q):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from wloop_b200 import measure as Mr
    from wloop_b200.replicas import Replicas
    try:
        rep = Replicas(backend="gloo", timeout_s=20)
        if mode == "run":
            head = Mr.dat_head(P, N[0])
            r = Mr.Run("rep", N, 3, P, first=1, last=9, step=1)
            res = Mr.run(r, out_dir, rep, measure=lambda nc: fake_wl(nc, head[0]))
            mx = rep.max(rank + 1.5)
            tot = rep.sum(len(res["configs"]))
            rep.close()
            q.put((rank, res["configs"], res.get("records"), mx, tot))
        else:  # "leave": rank 1 exits without joining the barrier
            if rank == 1:
                q.put((rank, "left"))
                q.close()
                q.join_thread()  # flush before leaving without clean-up
                os._exit(0)
            t0 = time.time()
            try:
                rep.barrier()
                q.put((rank, "barrier returned"))
            except Exception as e:  # noqa: BLE001
                q.put((rank, f"raised after {time.time() - t0:.1f}s: {type(e).__name__}"))
    except Exception as e:  # noqa: BLE001
        q.put((rank, f"error: {e!r}"))


def _spawn(world, out_dir, mode, wait_s=120):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_replica_main, args=(r, world, port, out_dir, mode, q))
          for r in range(world)]
    for p in ps:
        p.start()
    out = []
    try:
        for _ in range(world):
            out.append(q.get(timeout=wait_s))
    finally:
        for p in ps:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    return sorted(out, key=lambda x: x[0])


def test_two_replicas_gloo_merge_equals_single_process(tmp_path):
    out = _spawn(2, str(tmp_path / "rep"), "run")
    assert out[0][1] == [1, 3, 5, 7, 9] and out[1][1] == [2, 4, 6, 8]
    assert out[0][2] == 9  # rank 0 merged all records
    assert out[0][3] == out[1][3] == 2.5  # max over ranks
    assert out[0][4] == out[1][4] == 9
    head = M.dat_head(P, N[0])
    single = M.run(M.Run("rep", N, 3, P, first=1, last=9), str(tmp_path / "one"),
                   measure=lambda nc: fake_wl(nc, head[0]))
    assert single["configs"] == list(range(1, 10))
    a = open(tmp_path / "rep" / "rep.ms10.dat", "rb").read()
    b = open(tmp_path / "one" / "rep.ms10.dat", "rb").read()
    assert a == b


def test_replica_that_leaves_does_not_hang_the_other(tmp_path):
    out = _spawn(2, str(tmp_path), "leave", wait_s=90)
    assert out[1][1] == "left"
    assert out[0][1].startswith("raised"), out[0][1]


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
@pytest.mark.gpu
def test_run_on_gpu_matches_context_and_oracle(tmp_path):
    from tests import oracle as O
    from wloop_b200 import Context, generate_links
    r = M.Run("g", N, 0, P, first=1, last=3, precision="fp64", eps=0.25)
    fields = {nc: generate_links(N, 0, 100 + nc, 0.25) for nc in r.configs}
    M.run(r, str(tmp_path), source=lambda nc: fields[nc])
    h, ncs, wl = M.read(str(tmp_path / "g.ms10.dat"))
    assert list(ncs) == [1, 2, 3]
    with Context(N, 0, "fp64") as ctx:
        for k, nc in enumerate(ncs):
            ctx.upload(fields[nc])
            assert np.array_equal(ctx.measure(P), wl[k])
    u = O.hyp_links(N, 0, fields[2], *P.alpha_action, 1, P.proj_iter)
    ref = O.wloop_sum(N, 0, u, P)
    scale = np.maximum(np.abs(ref), 1.0)
    assert np.max(np.abs(wl[1] - ref) / scale) < 1e-12


@pytest.mark.gpu
def test_run_synthetic_on_gpu(tmp_path):
    from wloop_b200 import Context
    r = M.Run("s", N, 3, P, first=5, last=6, precision="mixed", eps=0.2)
    M.run(r, str(tmp_path))
    h, ncs, wl = M.read(str(tmp_path / "s.ms10.dat"))
    with Context(N, 3, "mixed") as ctx:
        ctx.generate(6, 0.2)
        assert np.array_equal(ctx.measure(P), wl[1])


def test_merge_refuses_a_short_rank_file(tmp_path):
    """A rank that failed part-way leaves fewer records than its share; rank 0
    then refuses to write the merged file (here with a fake two-rank group)."""
    head = M.dat_head(P, N[0])

    class Rank0:
        rank, world, local, device = 0, 2, 0, 0

        def barrier(self):
            pass
    # rank 1's file: head only, as a rank that died before its first record
    M.write_head(M.dat_path(str(tmp_path), "s", 1, 2), head)
    r = M.Run("s", N, 3, P, first=1, last=5)
    with pytest.raises(WlgError, match="rank 1 wrote 0 of its 2 records"):
        M.run(r, str(tmp_path), Rank0(), measure=lambda nc: fake_wl(nc, head[0]))
    assert not os.path.exists(tmp_path / "s.ms10.dat")
