#!/usr/bin/env python
"""Headline benchmark: Wilson-loop measurements (configs/s) at 32^3x64.

One step = one full measurement of one synthetic 32^3x64 configuration, the
work ms10's set_data does per configuration (main/ms10.c:633-646):
HYP2 smearing of all links, 6 APE levels (nss 0 10 10 10 10 10, alpha 0.5),
and the 6x6 Wilson-loop matrices for r <= 16, t <= 24 on every time slice.
The headline form is mixed precision (FP32 links / staples / line products,
FP64 projection and sums); the FP64 form runs the same workload and the
per-entry error of the mixed result against it is reported.

  value    configs/s with the input field resident in HBM (device-to-device
           restore of the unsmeared field at the start of each step)
  e2e      configs/s through the public API from a pinned host buffer: the
           FP64 su3_dble field (H2D) in, the wl_mat (D2H) out, every step;
           the next step's field is copied while the current one is
           measured (Context.prefetch / upload_prefetched)
  roofline the Wilson-loop contraction kernel (the dominant kernel), its
           algorithmic flops per launch over its CUDA-event time

Multi-GPU (torchrun): independent replicas, one configuration stream per
GPU, no collective on the data path ("scaling": "weak").

--impl reference times the reference algorithm's CPU implementation (the
FP64 oracle port, since the reference itself cannot be built here) on a
bounded sample of the same workload on all host cores.
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
    ap.add_argument("--lattice", default=None,
                    help="N0xN1xN2xN3 override for small profiling captures (not a bench line)")
    ap.add_argument("--workload", default="c3", choices=["c3", "c3b", "c4", "c5"],
                    help="c3: headline single configuration; c3b: 4 configurations of c3 in one "
                         "graph launch; c4: 64-configuration batch in one graph launch; c5: "
                         "serving loop with Poisson arrivals")
    ap.add_argument("--requests", type=int, default=100, help="c5: number of requests")
    ap.add_argument("--rate", type=float, default=20.0, help="c5: arrivals per second")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU side: bounded, stage-wise sample of the reference algorithm (oracle)
# ---------------------------------------------------------------------------
def cpu_sample(ns: int, nt: int, threads: int):
    """Times the FP64 oracle (the reference algorithm restated) on an
    ns^3 x nt lattice with the workload's per-site parameters: HYP once, one
    APE sweep, and the loop stage for r,t <= 4 with msl 6.  Every stage is
    linear in the volume, APE in the sweep count, and the reference's
    loop contraction costs the same per (r,t) pair (wloop.c:545-571), so
    t_config = (V/V_s) (t_hyp + 50 t_ape + (16*24/16) t_loop)."""
    from tests import oracle as O  # checker / baseline only
    from wloop_b200.api import WloopParms, generate_links
    from wloop_b200.workloads import C3
    O.set_threads(threads)
    n = (nt, ns, ns, ns)
    u = generate_links(n, 3, 3, 0.2)
    t0 = time.perf_counter()
    uh = O.hyp_links(n, 3, u, 1.0, 1.0, 0.5, 1, 4)
    t1 = time.perf_counter()
    O.ape_links(n, uh, 0.5, 1, 4, time=0, nsweeps=1)
    t2 = time.perf_counter()
    p = WloopParms(msl=6, nss=[0] * 6, mwlt=4, mwlr=4, alpha_ape=0.5, proj_iter=4)
    O.wloop_sum(n, 3, uh, p)
    t3 = time.perf_counter()
    c3 = C3.parms
    scale_v = C3.volume / float(nt * ns ** 3)
    sweeps = sum(c3.nss[:c3.msl])
    pairs = (c3.mwlr * c3.mwlt) / 16.0
    t_cfg = scale_v * ((t1 - t0) + sweeps * (t2 - t1) + pairs * (t3 - t2))
    sample = (f"oracle on {ns}^3x{nt} (1/{scale_v:.1f} of the volume): HYP once "
              f"{t1 - t0:.2f}s, one APE sweep {t2 - t1:.2f}s, loops r,t<=4 msl 6 {t3 - t2:.2f}s; "
              f"scaled by volume, {sweeps} sweeps and {pairs:.0f}x the (r,t) pairs")
    return 1.0 / t_cfg, t3 - t0, sample


def run_reference(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    times, samples = [], ""
    for i in range(args.warmup + args.steps):
        v, wall, samples = cpu_sample(12, 24, threads)
        if i >= args.warmup:
            times.append(1.0 / v)
    t = statistics.mean(times)
    value = 1.0 / t
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": "c3: 32^3x64 periodic, HYP2, APE 0.5 nss 0 10 10 10 10 10, "
                                   "msl 6, r<=16, t<=24", "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": samples},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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

    def timed_value(prec, steps, warmup, profile):
        ctx = Context(w.n, w.bc, prec, device=local)
        ctx.generate(w.seed + 1000 * rank, w.eps)
        ctx.snapshot()
        for _ in range(warmup):
            ctx.restore()
            ctx.measure(p)
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
            wl = ctx.measure(p)
        e1.record(ext)
        e1.synchronize()
        torch.cuda.synchronize(local)
        l1 = launch_count()
        ck = clocks.stop()
        barrier()
        ms = e0.elapsed_time(e1) / steps
        kt = {k: ctx.kernel_time(k) for k in ("hyp", "ape", "plaq", "lines", "contract", "reduce")}
        ctx.set_profiling(False)
        return ctx, ms, wl, kt, ck, l1 - l0

    # ---- headline precision: device-resident value ----
    ctx, ms, wl_main, kt, clocks, launches = timed_value(args.precision, args.steps, args.warmup,
                                                         True)
    ms_max = barrier_max(ms)
    value = world * 1000.0 / ms_max

    # ---- e2e through the public API from pinned host memory ----
    e2e = None
    if not args.skip_e2e:
        host = torch.empty((w.volume * 4 * 18,), dtype=torch.float64, pin_memory=True)
        hnp = host.numpy().view(np.complex128).reshape(w.volume, 4, 3, 3)
        ctx.restore()
        hnp[...] = ctx.download()
        ctx.prefetch(hnp)
        ctx.upload_prefetched()
        ctx.measure(p)  # warm the staging buffer
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
            out = ctx.measure(p)
        e1.record(ext)
        e1.synchronize()
        barrier()
        ems = barrier_max(e0.elapsed_time(e1) / args.steps)
        e2e = {"value": world * 1000.0 / ems, "unit": UNIT,
               "h2d_bytes_per_step": int(hnp.nbytes), "d2h_bytes_per_step": int(out.nbytes),
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

    # ---- roofline of the dominant kernel (contraction) ----
    c_ms, c_n = kt["contract"]
    per_launch_ms = c_ms / max(1, c_n)
    # the contraction launches also carry the spatial line step of the next R
    flops_per_launch = (fl["contract"] + fl["lines"]) / p.mwlr
    achieved = flops_per_launch / (per_launch_ms * 1e-3) / 1e12
    peak = peak_tflops(args.precision, local)
    traffic = load_traffic().get(args.precision)
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
    bytes_per_launch = link_b * vol * ((3 * p.msl + 1) + 6 * p.msl * (p.mwlr - 1) / p.mwlr)
    hbm_ach = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    roof = {"kernel": "k_contract4 (loop contraction with the fused spatial line step)",
            "bound": "fp32" if args.precision == "mixed" else "fp64",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
            "peak_source": "vector FMA probe measured in this run (wlg_peak_flops; of measured); "
                           "the kernel is bound by CUDA-core FMA throughput, not by HBM or "
                           "tensor cores (3x3 complex products have no tensor-core form), "
                           "and MEASURED_PEAKS.json has no CUDA-core peak",
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

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        threads = os.cpu_count() or 1
        v, wall, sample = cpu_sample(16, 32, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}

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
                "algorithmic_flops_per_config": fl["total"]}
        print(json.dumps(line), flush=True)
    rep.close()


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


def run_serve(args):
    """c5: measurement requests with Poisson arrivals (rate --rate) over the
    volumes {16^3x32, 24^3x48, 32^3x64, 48^3x96}, eps ~ U[0.15,0.35], bc
    open/periodic 50/50, HYP2 + 4 APE levels, r,t <= Ns/2; p50/p99 latency and
    throughput for the mixed and the FP64 forms."""
    import random
    from wloop_b200.api import Server, aux_uniform
    from wloop_b200.workloads import serving_request
    out = {"metric": "serving: p50/p99 latency (ms) and configs/s, Poisson arrivals",
           "unit": "configs/s", "n_gpus": 1, "higher_is_better": True, "data": "synthetic",
           "requests": args.requests, "rate_per_s": args.rate, "forms": {}}
    for prec, nreq in (("mixed", args.requests), ("fp64", max(10, args.requests // 3))):
        reqs = [serving_request(i) for i in range(nreq)]
        t = 0.0
        arrivals = []
        for i in range(nreq):  # exponential inter-arrival times from the seeded stream
            u = aux_uniform(5000, i, 7)
            t += -math.log(1.0 - u) / args.rate
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
            st = s.stats()
        mix = {}
        for w in reqs:
            key = "x".join(str(v) for v in (w.n[1], w.n[1], w.n[1], w.n[0]))
            mix[key] = mix.get(key, 0) + 1
        out["forms"][prec] = {"requests": nreq, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
                              "configs_per_s": st["throughput"], "batches": st["batches"],
                              "failed": st["failed"], "volume_mix": mix}
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
    if args.workload == "c5":
        run_serve(args)
        return
    run_ours(args, rank, world, local)


if __name__ == "__main__":
    main()
