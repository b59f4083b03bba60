#!/usr/bin/env python
"""Headline benchmark: Wilson-loop measurements (configs/s) at 32^3x64.

One step = one full measurement of one synthetic 32^3x64 configuration, the
work ms10's set_data does per configuration (main/ms10.c:633-646):
HYP2 smearing of all links, 6 APE levels (nss 0 10 10 10 10 10, alpha 0.5),
and the 6x6 Wilson-loop matrices for r <= 16, t <= 24 on every time slice,
plus the plaquette after every smearing level.
The headline form is mixed precision (FP32 links / staples / line products,
FP64 projection and sums); the FP64 form runs the same workload and the
per-entry error of the mixed result against it is reported.

  value    configs/s with the input field resident in HBM (device-to-device
           restore of the unsmeared field at the start of each step)
  e2e      configs/s through the public API from a pinned host buffer: the
           FP64 su3_dble field (H2D) in, the wl_mat and plaquettes (D2H)
           out, every step;
           the next step's field is copied while the current one is
           measured (Context.prefetch / upload_prefetched)
  roofline the Wilson-loop contraction kernel (the dominant kernel), its
           algorithmic flops per launch over its CUDA-event time

Multi-GPU (torchrun): independent replicas, one configuration stream per
GPU, no collective on the data path ("scaling": "weak").

cpu_baseline: the oracle (the reference algorithm restated, OpenMP) on all
host threads, on full-size pieces of the workload; c1_measured_pair: the 8^4
workload measured whole by the GPU and by the reference itself.

--impl reference times the reference's own CPU implementation: its modules
compiled from source (oracle/_ref), as one-core replicas on all host cores
(without MPI the reference runs one process per core), each step one
full-size APE sweep in every replica, with HYP and the loop stage timed at
full size in two further replicas meanwhile.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "configs/s at 32^3x64, mixed vs FP64 GPU at <=1e-6 rel err; p50/p99 latency"
UNIT = "configs/s"
# HBM copy bandwidth used when no measured peak file is present (GB/s)
HBM_FALLBACK_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--skip-fp64", action="store_true", help="do not run the FP64 comparison")
    ap.add_argument("--skip-cpu", action="store_true", help="do not time the CPU baseline")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--forms", default="", help="comma-separated contraction forms to time "
                    "beside the default (mixed), e.g. 8,9")
    ap.add_argument("--lattice", default=None,
                    help="N0xN1xN2xN3 override for small profiling captures (not a bench line)")
    ap.add_argument("--workload", default="c3", choices=["c3", "c3b", "c4", "c5", "c5sweep"],
                    help="c3: headline single configuration; c3b: 4 configurations of c3 in one "
                         "graph launch; c4: 64-configuration batch in one graph launch; c5: "
                         "serving loop with Poisson arrivals")
    ap.add_argument("--requests", type=int, default=100, help="c5: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="c5: arrivals per second")
    ap.add_argument("--sweep-rates", default="1,2,3,4,6", help="c5sweep: arrival rates")
    ap.add_argument("--sweep-requests", type=int, default=120, help="c5sweep: requests per rate")
    ap.add_argument("--stable-p99-s", type=float, default=10.0,
                    help="c5sweep: p99 latency bound of a stable rate (seconds)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU side: the reference itself (oracle/_ref) and the oracle, timed on full-
# size pieces of the workload.  Nothing here loads the product library: the
# inputs come from the oracle's copy of the field generator.
# ---------------------------------------------------------------------------
class _Parms:
    """The workload's wloop parameters, without importing the product package
    (whose import loads libwloop_b200.so)."""

    def __init__(self, msl, nss, mwlt, mwlr):
        self.msl, self.nss, self.mwlt, self.mwlr = msl, list(nss), mwlt, mwlr
        self.op_smear, self.alpha_action, self.alpha_ape = 0, (1.0, 1.0, 0.5), 0.5
        self.alpha_hyp, self.proj_iter, self.proj = (0.0, 0.0), 4, 1


C3_N, C3_BC, C3_SEED, C3_EPS = (64, 32, 32, 32), 3, 3, 0.2
C3_P = _Parms(6, [0, 10, 10, 10, 10, 10], 24, 16)
C1_N, C1_BC, C1_SEED, C1_EPS = (8, 8, 8, 8), 3, 1, 0.3
C1_P = _Parms(4, [0, 5, 5, 5], 4, 4)
C3_DESC = ("c3: 32^3x64 periodic, eps 0.2, HYP2 (1,1,0.5) proj 4, APE 0.5 nss 0 10 10 10 10 10, "
           "msl 6, r<=16, t<=24")


def _loop_piece(p, mwlt):
    """wloop_sum parameters of one loop piece: all msl levels with no sweeps
    (the smearing is timed on its own), r = 1, t = 1..mwlt."""
    return _Parms(p.msl, [0] * p.msl, mwlt, 1)


def _piece_worker(mwlt, path, n, bc, p, q):
    """Full-size pieces of the reference in their own process: hyp_links once,
    then the loop stage for r = 1, t = 1..mwlt on the HYP-smeared field.
    Puts {name: seconds}."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from tests import refimpl as R
    ref = R.Ref(n)
    ref.set_field(bc, np.load(path, mmap_mode="r"))
    out = {}
    t0 = time.perf_counter()
    ref.hyp_links(*p.alpha_action, p.proj, p.proj_iter)
    out[f"hyp_{mwlt}"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    ref.wloop_sum(_loop_piece(p, mwlt))
    out[f"loops_t{mwlt}"] = time.perf_counter() - t0
    q.put(out)


def _ape_worker(path, n, bc, p, nsteps, barrier, q):
    """One replica of the reference: nsteps spatial APE sweeps of the full
    field, each started together with the other replicas' (barrier).  Puts
    the list of sweep times."""
    sys.path.insert(0, ROOT)
    import numpy as np
    from tests import refimpl as R
    ref = R.Ref(n)
    ref.set_field(bc, np.load(path, mmap_mode="r"))
    ts = []
    for _ in range(nsteps):
        barrier.wait(timeout=600)  # a replica that died breaks the barrier
        t0 = time.perf_counter()
        ref.ape_links(p.alpha_ape, p.proj, p.proj_iter, time=0, nsweeps=1)
        ts.append(time.perf_counter() - t0)
    q.put(ts)


def _mem_available_gb():
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) / 1e6
    except OSError:
        pass
    return 0.0


def _reference_c1(reps):
    """The 8^4 workload measured whole by the reference: seconds per
    configuration (ms10's set_data: hyp_links + wloop_sum)."""
    from tests import oracle as O
    from tests import refimpl as R
    ref = R.Ref(C1_N)
    u = O.generate_links(C1_N, C1_BC, C1_SEED, C1_EPS)
    ts = []
    for _ in range(reps):
        ref.set_field(C1_BC, u)
        t0 = time.perf_counter()
        ref.measure(C1_P)
        ts.append(time.perf_counter() - t0)
    return statistics.median(ts)


def run_reference(args, rank):
    """The reference's own CPU implementation (oracle/_ref: its modules built
    from source) on the 32^3x64 workload, on the host's cores.  Without MPI
    the reference runs one process per core, so the host runs it as
    independent replicas, one configuration stream each.  Every piece runs at
    the full size and under the load of all the replicas: each step is one
    spatial APE sweep (the ms10 run does 50 per configuration) in every APE
    replica at once; two further replicas run HYP and the loop stage for
    (r=1, t=1) and for (r=1, t=1,2) meanwhile.  Per replica a configuration
    takes t_config = t_hyp + 50 t_ape + (t_fixed + 384 t_pair), with t_pair =
    t(t<=2) - t(t<=1) and t_fixed = max(0, t(t<=1) - t_pair) (the reference's loop
    stage costs the same for every (r,t) pair at fixed msl, wloop.c:545-571;
    r <= 16, t <= 24 is 384 pairs), and the host's configs/s is the number of
    replicas over t_config.  The replica count is the core count, lowered if
    the host memory would not hold them (about 5 GB per APE replica, 22 GB
    per loop replica)."""
    if rank != 0:
        return
    import multiprocessing as mp
    import tempfile
    import numpy as np
    from tests import oracle as O
    from tests import refimpl as R
    p = C3_P
    if not R.available(C3_N):
        print(json.dumps({"impl": "reference", "unavailable":
                          "oracle/_ref was not built for 64x32x32x32 (make -C oracle ref)"}))
        return
    cores = os.cpu_count() or 1
    mem = _mem_available_gb()
    n_ape = max(1, min(cores - 2, int((mem - 2 * 22 - 6) // 5)))
    wall0 = time.perf_counter()
    O.set_threads(cores)
    tmpdir = tempfile.mkdtemp(prefix="wlref_")
    path = os.path.join(tmpdir, "c3_field.npy")
    np.save(path, O.generate_links(C3_N, C3_BC, C3_SEED, C3_EPS))
    ctx = mp.get_context("spawn")
    q_piece, q_ape = ctx.Queue(), ctx.Queue()
    nsteps = args.warmup + args.steps
    barrier = ctx.Barrier(n_ape)
    procs = [ctx.Process(target=_piece_worker, args=(k, path, C3_N, C3_BC, p, q_piece))
             for k in (1, 2)]
    procs += [ctx.Process(target=_ape_worker, args=(path, C3_N, C3_BC, p, nsteps, barrier, q_ape))
              for _ in range(n_ape)]
    for pr in procs:
        pr.start()
    import queue
    try:
        # every piece is minutes of work; an hour means a replica died
        ape = [q_ape.get(timeout=3600) for _ in range(n_ape)]
        pieces = {}
        for _ in range(2):
            pieces.update(q_piece.get(timeout=3600))
    except queue.Empty:
        for pr in procs:
            if pr.is_alive():
                pr.terminate()
        print(json.dumps({"impl": "reference", "unavailable":
                          "a replica of the reference did not report (died or ran out of memory)"}))
        return
    finally:
        os.remove(path)
        os.rmdir(tmpdir)
    for pr in procs:
        pr.join()
    # a step ends when the slowest replica's sweep ends
    steps = [max(ts[i] for ts in ape) for i in range(args.warmup, nsteps)]
    t_ape = statistics.mean(steps)
    pieces["hyp"] = 0.5 * (pieces["hyp_1"] + pieces["hyp_2"])
    t_c1 = _reference_c1(3)
    sweeps = sum(p.nss[:p.msl])
    pairs = p.mwlr * p.mwlt
    t_pair = pieces["loops_t2"] - pieces["loops_t1"]
    # the one-time part of the loop stage, never below zero (the two loop
    # pieces run in different replicas and their load can differ a little)
    t_fixed = max(0.0, pieces["loops_t1"] - t_pair)
    t_cfg = pieces["hyp"] + sweeps * t_ape + t_fixed + pairs * t_pair
    replicas = n_ape + 2
    value = replicas / t_cfg
    sample = (f"the reference's modules built from source (oracle/_ref), {replicas} one-core "
              f"replicas at once on {cores} cores, at the full 32^3x64 size: one spatial APE "
              f"sweep {t_ape:.2f} s ({n_ape} replicas in step, mean of {len(steps)} timed "
              f"steps; 50 per configuration); hyp_links {pieces['hyp']:.1f} s; loop stage "
              f"r=1,t=1 {pieces['loops_t1']:.1f} s and r=1,t<=2 {pieces['loops_t2']:.1f} s (per "
              f"(r,t) pair {t_pair:.1f} s, 384 pairs); {t_cfg:.0f} s per configuration and "
              f"replica, configs/s = replicas / that")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_ape * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": C3_DESC, "parallelism": f"{replicas} replicas of the "
                       f"one-process reference (no MPI), one per core"},
            "step": f"one full-size spatial APE sweep (ape_spatial_links) in each of {n_ape} "
                    f"replicas at once",
            "value_kind": "estimate from full-size pieces measured under the load of all replicas",
            "pieces_s": {"hyp": pieces["hyp"], "hyp_runs": [pieces["hyp_1"], pieces["hyp_2"]],
                         "ape_sweep": t_ape,
                         "loops_r1_t1": pieces["loops_t1"], "loops_r1_t2": pieces["loops_t2"],
                         "per_pair": t_pair, "fixed": t_fixed, "config_per_replica": t_cfg},
            "replicas": replicas, "host_memory_available_gb": mem,
            "wall_s": time.perf_counter() - wall0,
            "c1_measured": {"workload": "c1: 8^4 periodic, eps 0.3, HYP2, APE 0.5 nss 0 5 5 5, "
                                        "msl 4, r,t<=4", "seconds_per_config": t_c1,
                            "configs_per_s_one_core": 1.0 / t_c1,
                            "kind": "reference, whole measurement, one core"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": replicas, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_sample(threads: int):
    """The oracle (the reference algorithm restated, OpenMP over sites) on
    full-size pieces of the 32^3x64 workload on all host threads: hyp once,
    one spatial APE sweep, the loop stage for (r=1,t=1) and (r=1,t<=2);
    configs/s estimated as in run_reference."""
    from tests import oracle as O
    p = C3_P
    O.set_threads(threads)
    u = O.generate_links(C3_N, C3_BC, C3_SEED, C3_EPS)
    t0 = time.perf_counter()
    uh = O.hyp_links(C3_N, C3_BC, u, *p.alpha_action, p.proj, p.proj_iter)
    t1 = time.perf_counter()
    O.ape_links(C3_N, uh, p.alpha_ape, p.proj, p.proj_iter, time=0, nsweeps=1)
    t2 = time.perf_counter()
    O.wloop_sum(C3_N, C3_BC, uh, _loop_piece(p, 1))
    t3 = time.perf_counter()
    O.wloop_sum(C3_N, C3_BC, uh, _loop_piece(p, 2))
    t4 = time.perf_counter()
    sweeps = sum(p.nss[:p.msl])
    t_pair = (t4 - t3) - (t3 - t2)
    t_fixed = max(0.0, (t3 - t2) - t_pair)
    t_cfg = (t1 - t0) + sweeps * (t2 - t1) + t_fixed + p.mwlr * p.mwlt * t_pair
    sample = (f"oracle on {threads} threads at the full 32^3x64 size: HYP {t1 - t0:.2f} s, one "
              f"APE sweep {t2 - t1:.3f} s (x{sweeps}), loop stage r=1,t=1 {t3 - t2:.2f} s and "
              f"r=1,t<=2 {t4 - t3:.2f} s (x{p.mwlr * p.mwlt} pairs); estimated from these "
              f"measured pieces")
    return 1.0 / t_cfg, t4 - t0, sample


# ---------------------------------------------------------------------------
# GPU side
# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for nm, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def gram_flops_per_launch(w):
    """Flops of one banded Gram launch: every (x0, T, s1, s2) is a dot product
    over 3 directions x vs sites x 18 components."""
    p = w.parms
    vs = w.volume // w.n[0]
    return 2.0 * w.n[0] * p.mwlt * p.msl * p.msl * 3 * vs * 18


def load_traffic():
    p = os.path.join(ROOT, "profiles", "contract_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return {}


def run_ours(args, rank, world, local):
    import numpy as np
    import torch
    from wloop_b200.api import Context, launch_count, peak_tflops
    from wloop_b200.workloads import C3, flops_per_config

    from wloop_b200.replicas import Replicas
    rep = Replicas()
    barrier_max, barrier = rep.max, rep.barrier
    local = rep.device  # this rank's GPU

    w = C3
    if args.lattice:
        import dataclasses
        n = tuple(int(x) for x in args.lattice.split("x"))
        pp = dataclasses.replace(w.parms, mwlt=min(w.parms.mwlt, n[0] // 2 + 1),
                                 mwlr=min(w.parms.mwlr, n[1] // 2 + 1))
        w = dataclasses.replace(w, n=n, parms=pp)
    p = w.parms
    fl = flops_per_config(w)

    def timed_value(prec, steps, warmup, profile, variant=0):
        ctx = Context(w.n, w.bc, prec, device=local)
        if variant:
            ctx.set_contract_tuning(variant=variant)
        ctx.generate(w.seed + 1000 * rank, w.eps)
        ctx.snapshot()
        for _ in range(warmup):
            ctx.restore()
            ctx.measure(p, plaq=True)
        ext = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ctx.reset_kernel_times()
        ctx.set_profiling(profile)
        clocks = ClockSampler(local)
        barrier()
        torch.cuda.synchronize(local)
        clocks.start()
        l0 = launch_count()
        e0.record(ext)
        wl = None
        for _ in range(steps):
            ctx.restore()
            wl, _ = ctx.measure(p, plaq=True)
        e1.record(ext)
        e1.synchronize()
        torch.cuda.synchronize(local)
        l1 = launch_count()
        ck = clocks.stop()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        kt = {k: ctx.kernel_time(k)
              for k in ("hyp", "ape", "plaq", "gauge", "lines", "contract", "reduce")}
        ctx.set_profiling(False)
        return ctx, ms, wl, kt, ck, l1 - l0

    # ---- headline precision: device-resident value ----
    ctx, ms, wl_main, kt, clocks, launches = timed_value(args.precision, args.steps, args.warmup,
                                                         True)
    ms_max = barrier_max(ms)
    value = world * 1000.0 / ms_max
    form = ctx.contract_form

    # ---- e2e through the public API from pinned host memory ----
    e2e = None
    if not args.skip_e2e:
        host = torch.empty((w.volume * 4 * 18,), dtype=torch.float64, pin_memory=True)
        hnp = host.numpy().view(np.complex128).reshape(w.volume, 4, 3, 3)
        ctx.restore()
        hnp[...] = ctx.download()
        ctx.prefetch(hnp)
        ctx.upload_prefetched()
        ctx.measure(p, plaq=True)  # warm the staging buffer
        ext = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize(local)
        # a measurement stream as a driver runs it: the next configuration's
        # host-to-device copy (on the context's copy stream) overlaps the
        # current measurement; every step copies its 1.2 GB field in and its
        # wl_mat out inside the timed region
        e0.record(ext)
        ctx.prefetch(hnp)
        for i in range(args.steps):
            ctx.upload_prefetched()
            if i + 1 < args.steps:
                ctx.prefetch(hnp)
            out, pl = ctx.measure(p, plaq=True)
        e1.record(ext)
        e1.synchronize()
        barrier()
        ems = barrier_max(e0.elapsed_time(e1) / args.steps)
        e2e = {"value": world * 1000.0 / ems, "unit": UNIT,
               "h2d_bytes_per_step": int(hnp.nbytes),
               "d2h_bytes_per_step": int(out.nbytes + pl.nbytes),
               "pipelined": "next field's H2D copy overlaps the current measurement"}
    ctx.close()

    # ---- FP64 form and the mixed-vs-FP64 error ----
    fp64 = None
    if not args.skip_fp64 and args.precision == "mixed":
        c64, ms64, wl64, kt64, _, _ = timed_value("fp64", max(2, min(args.steps, 3)), 1, True)
        c64.close()
        ms64 = barrier_max(ms64)
        zero = wl64 == 0.0
        rel = np.abs(wl_main - wl64)[~zero] / np.abs(wl64)[~zero]
        fp64 = {"value": world * 1000.0 / ms64, "ms_per_step": ms64,
                "mixed_over_fp64": ms64 / ms_max,
                "max_rel_err": float(rel.max()),
                "frac_entries_le_1e-6": float(np.mean(rel <= 1e-6)),
                "median_rel_err": float(np.median(rel)),
                "contract_ms_per_launch": kt64["contract"][0] / max(1, kt64["contract"][1])}

    # ---- the contraction forms side by side (same run, same clocks) ----
    forms = None
    if args.forms and args.precision == "mixed":
        forms = {}
        for v in (int(x) for x in args.forms.split(",")):
            cv, msv, wlv, ktv, _, _ = timed_value("mixed", max(2, min(args.steps, 3)), 1, True, v)
            cv.close()
            forms[str(v)] = {"ms_per_step": barrier_max(msv),
                             "contract_ms_per_launch": ktv["contract"][0] / max(1, ktv["contract"][1]),
                             "max_abs_diff_vs_default": float(np.abs(wlv - wl_main).max())}

    # ---- roofline of the dominant kernel (contraction) ----
    c_ms, c_n = kt["contract"]
    per_launch_ms = c_ms / max(1, c_n)
    if form == 11:
        # the banded Gram product: 2 N0 mwlt msl^2 (3 vs 18) flops per R
        flops_per_launch = gram_flops_per_launch(w)
    else:
        # the contraction launches also carry the spatial line step of the next R
        flops_per_launch = (fl["contract"] + fl["lines"]) / p.mwlr
    achieved = flops_per_launch / (per_launch_ms * 1e-3) / 1e12
    peak = peak_tflops(args.precision, local)
    peak_src = "vector FMA probe measured in this run (wlg_peak_flops, fma.rn.f64; of measured)"
    peaks_probe = None
    if args.precision == "mixed":
        # the kernel issues packed two-lane FMAs: the FP32 roof is the higher
        # of the scalar and the packed probe
        p_scalar, p_x2 = peak, peak_tflops("f32x2", local)
        peaks_probe = {"fma.rn.f32": p_scalar, "fma.rn.f32x2": p_x2}
        peak = max(p_scalar, p_x2)
        peak_src = ("vector FMA probe measured in this run (wlg_peak_flops): the higher of "
                    "scalar fma.rn.f32 and packed fma.rn.f32x2 chains; of measured")
    traffic = load_traffic().get(args.precision + ("_gram" if form == 11 else ""))
    peaks_file = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm, hbm_src = None, None
    if os.path.exists(peaks_file):
        with open(peaks_file) as f:
            hbm = json.load(f).get("hbm_gbs")
        hbm_src = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if not hbm:
        # an earlier STREAM-style copy measurement on B200s of this kind
        hbm, hbm_src = HBM_FALLBACK_GBS, "6650 GB/s earlier B200 copy measurement (of fallback)"

    # algorithmic bytes of one launch: its lines of length R and temporal links
    # ((3 msl + 1) V links) plus the fused line step's level links in and new
    # lines out (2 x 3 msl V, for 15 of the 16 launches)
    link_b = 72 if args.precision == "mixed" else 144
    vol = w.volume
    if form == 11:
        # its A lines (N0 slices) and B lines (N0 + mwlt slices, periodic), once
        nu = w.n[0] + (p.mwlt if w.bc != 0 else 0)
        bytes_per_launch = link_b * (w.n[0] + nu) * (vol // w.n[0]) * 3 * p.msl
        kname = "k_gram (banded Gram product of the temporal-gauge lines)"
    else:
        bytes_per_launch = link_b * vol * ((3 * p.msl + 1) + 6 * p.msl * (p.mwlr - 1) / p.mwlr)
        kname = "k_contract4 (loop contraction with the fused spatial line step)"
    hbm_ach = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    roof = {"kernel": kname, "contract_form": form,
            "bound": "fp32" if args.precision == "mixed" else "fp64",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": peak_src + "; the kernel is bound by CUDA-core FMA throughput, not "
                           "by HBM (its FP32 dot products need more precision than one "
                           "TF32/BF16 tensor-core pass gives), and MEASURED_PEAKS.json has no "
                           "CUDA-core peak",
            "peak_probes_tflops": peaks_probe,
            "flops_per_launch": flops_per_launch, "ms_per_launch": per_launch_ms,
            "traffic": traffic,
            "hbm": {"achieved": hbm_ach, "peak": hbm, "unit": "GB/s",
                    "frac": (hbm_ach / hbm) if hbm else None,
                    "algorithmic_bytes_per_launch": bytes_per_launch,
                    "traffic_frac": (traffic / (per_launch_ms * 1e-3) / 1e9 / hbm)
                    if (traffic and hbm) else None,
                    "peak_source": hbm_src}}
    total_ms = sum(v[0] for v in kt.values())
    shares = {k: round(v[0] / total_ms, 4) for k, v in kt.items() if total_ms > 0}

    # ---- mixed result against the FP64 oracle's fixture (two time slices) ----
    vs_oracle = None
    fx = os.path.join(ROOT, "tests", "golden", "c3_32x32x32x64_periodic.npz")
    if not args.lattice and args.precision == "mixed" and os.path.exists(fx):
        f = np.load(fx)
        got = wl_main.reshape(w.n[0], -1)[f["x0"]]
        nz = f["wl"] != 0.0
        rel = np.abs(got - f["wl"])[nz] / np.abs(f["wl"])[nz]
        vs_oracle = {"max_rel_err": float(rel.max()), "median_rel_err": float(np.median(rel)),
                     "entries": int(rel.size), "time_slices": [int(x) for x in f["x0"]]}

    cpu = None
    c1 = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        v, wall, sample = cpu_sample(threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}
        c1 = c1_pair(local)


    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32+f64" if args.precision == "mixed" else "f64",
                "data": "synthetic",
                "config": {"workload": "c3: 32^3x64 periodic, eps 0.2, HYP2 (1,1,0.5) proj 4, "
                                       "APE 0.5 nss 0 10 10 10 10 10, msl 6, r<=16, t<=24",
                           "precision": args.precision, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (field 151-302 MB, level store 1.9-3.8 GB)"},
                "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
                "gpu_launches": launches, "fp64_form": fp64, "kernel_share": shares,
                "mixed_vs_oracle_fixture": vs_oracle, "c1_measured_pair": c1,
                "contract_forms": forms,
                "algorithmic_flops_per_config": fl["total"]}
        print(json.dumps(line), flush=True)
    rep.close()


def c1_pair(device):
    """The 8^4 workload measured whole on both sides: the GPU through the
    public API (host field in, wl_mat and plaquettes out, per configuration)
    in both forms, and the reference itself (oracle/_ref) on one core."""
    import numpy as np
    from wloop_b200.api import Context, generate_links
    from wloop_b200.workloads import C1
    out = {"workload": "c1: 8^4 periodic, eps 0.3, HYP2, APE 0.5 nss 0 5 5 5, msl 4, r,t<=4"}
    u = generate_links(C1.n, C1.bc, C1.seed, C1.eps)
    for prec in ("mixed", "fp64"):
        with Context(C1.n, C1.bc, prec, device=device) as c:
            for _ in range(3):
                c.upload(u)
                c.measure(C1.parms, plaq=True)
            reps = 50
            t0 = time.perf_counter()
            for _ in range(reps):
                c.upload(u)
                c.measure(C1.parms, plaq=True)
            out[f"gpu_{prec}_configs_per_s"] = reps / (time.perf_counter() - t0)
    from tests import refimpl as R
    if R.available(C1.n):
        t = _reference_c1(3)
        out["reference_configs_per_s"] = 1.0 / t
        out["reference_cores"] = 1
        out["gpu_mixed_over_reference"] = out["gpu_mixed_configs_per_s"] * t
    return out


def run_batch(args):
    """c4: 48 x 16^3x32 + 16 x 24^3x48, HYP2 + 4 APE levels, r,t <= Ns/2, mixed
    precision, all 64 configurations in one CUDA-graph launch per step."""
    import numpy as np
    import torch
    from wloop_b200.api import Batch, launch_count
    from wloop_b200.autotune import tune_batch
    from wloop_b200.workloads import batch_workloads, flops_per_config
    if args.workload == "c3b":
        import dataclasses
        from wloop_b200.workloads import C3
        ws = [dataclasses.replace(C3, seed=C3.seed + i) for i in range(4)]
        metric = "configs/s, 4 x 32^3x64 (c3) in one graph launch"
        desc = ("c3 batch: 4 x 32^3x64 periodic, HYP2, APE 0.5 nss 0 10 10 10 10 10, msl 6, "
                "r<=16, t<=24, one graph launch per step")
    else:
        ws = batch_workloads()
        metric = "configs/s, 64-configuration batch (48 x 16^3x32 + 16 x 24^3x48)"
        desc = "c4 batch, HYP2 + APE 0.5 nss 0 5 5 5, r,t <= Ns/2, one graph launch per step"
    prec = args.precision
    b = Batch([(w.n, w.bc, w.parms) for w in ws], prec)
    b.generate([w.seed for w in ws], [w.eps for w in ws])
    shape = tune_batch(b)
    b.snapshot()
    for _ in range(args.warmup):
        b.restore()
        b.run()
    ext = torch.cuda.ExternalStream(b.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    clocks = ClockSampler(0)
    clocks.start()
    l0 = launch_count()
    e0.record(ext)
    for _ in range(args.steps):
        b.restore()
        b.run()
    e1.record(ext)
    e1.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1) / args.steps
    _, kern = b.stats()
    flops = sum(flops_per_config(w)["total"] for w in ws)
    line = {"metric": metric,
            "value": len(ws) * 1000.0 / ms, "unit": "configs/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if prec == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": desc, "precision": prec,
                       "contract_shape_G_SB_block_nCB": list(shape),
                       "device_bytes": b.device_bytes},
            "kernels_per_graph": kern, "gpu_launches_device_side": kern * args.steps,
            "host_launch_calls": launch_count() - l0,
            "algorithmic_tflops": flops / (ms * 1e-3) / 1e12, "clocks": ck}
    b.close()
    print(json.dumps(line), flush=True)


def _serve_once(prec, nreq, rate, seed=5000):
    """One serving run: nreq c5 requests (volumes from {16^3x32, 24^3x48,
    32^3x64, 48^3x96}, eps ~ U[0.15,0.35], bc 50/50 open/periodic, HYP2 + 4 APE
    levels, r,t <= Ns/2) with Poisson arrivals at `rate` per second."""
    from wloop_b200.api import Server, aux_uniform
    from wloop_b200.workloads import serving_request
    reqs = [serving_request(i, seed) for i in range(nreq)]
    t = 0.0
    arrivals = []
    for i in range(nreq):  # exponential inter-arrival times from the seeded stream
        u = aux_uniform(seed, i, 7)
        t += -math.log(1.0 - u) / rate
        arrivals.append(t)
    with Server(max_inflight=3, max_batch=8, mem_fraction=0.85) as s:
        t0 = time.perf_counter()
        ids = []
        for w, ta in zip(reqs, arrivals):
            dt = ta - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            ids.append(s.submit(w.n, w.bc, w.parms, prec, seed=w.seed, eps=w.eps))
        for i in ids:
            s.wait(i)
        wall = time.perf_counter() - t0
        st = s.stats()
    mix = {}
    for w in reqs:
        key = "x".join(str(v) for v in (w.n[1], w.n[1], w.n[1], w.n[0]))
        mix[key] = mix.get(key, 0) + 1
    return {"requests": nreq, "rate_per_s": rate, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "configs_per_s": st["throughput"], "batches": st["batches"], "failed": st["failed"],
            "arrival_span_s": arrivals[-1], "wall_s": wall, "volume_mix": mix}


def run_serve(args):
    """c5: measurement requests with Poisson arrivals (rate --rate) over the
    volumes {16^3x32, 24^3x48, 32^3x64, 48^3x96}, eps ~ U[0.15,0.35], bc
    open/periodic 50/50, HYP2 + 4 APE levels, r,t <= Ns/2; p50/p99 latency and
    throughput for the mixed and the FP64 forms (the same --requests each).
    --workload c5sweep adds, per form, runs at increasing arrival rates
    (--sweep-rates, --sweep-requests each): the saturating throughput is the
    completion rate at the highest rate, and the highest stable rate is the
    highest swept rate whose completion rate keeps up with the arrivals (at
    least 95 %) with p99 below --stable-p99-s."""
    out = {"metric": "serving: p50/p99 latency (ms) and configs/s, Poisson arrivals",
           "unit": "configs/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
           "requests": args.requests, "rate_per_s": args.rate, "forms": {}}
    for prec in ("mixed", "fp64"):
        out["forms"][prec] = _serve_once(prec, args.requests, args.rate)
    if args.workload == "c5sweep":
        rates = [float(x) for x in args.sweep_rates.split(",")]
        out["sweep"] = {}
        for prec in ("mixed", "fp64"):
            runs = [_serve_once(prec, args.sweep_requests, r) for r in rates]
            stable = [r["rate_per_s"] for r in runs
                      if r["configs_per_s"] >= 0.95 * r["requests"] / r["arrival_span_s"]
                      and r["p99_ms"] <= 1e3 * args.stable_p99_s]
            out["sweep"][prec] = {"runs": runs,
                                  "saturating_configs_per_s": max(r["configs_per_s"] for r in runs),
                                  "highest_stable_rate_per_s": max(stable) if stable else None,
                                  "stable_rule": f"completions >= 95% of arrivals per second and "
                                                 f"p99 <= {args.stable_p99_s} s"}
    out["value"] = out["forms"]["mixed"]["configs_per_s"]
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload in ("c3b", "c4"):
        run_batch(args)
        return
    if args.workload in ("c5", "c5sweep"):
        run_serve(args)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
