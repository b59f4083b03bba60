"""Autotuner for the contraction kernel's shape (the dominant kernel).

A shape is (G bottom levels per thread, SB top levels per reduction, threads
per block, column blocks per (x0, level group)); SB 9 and 11 mark the ninth
and the temporal-gauge forms, and a context is timed over its whole loop
stage (gauge transformation, line steps, contraction, reduction).  The tuner times every
candidate on the caller's own data -- a Context (one lattice) or a Batch
(many) -- through the C ABI, keeps the fastest, and caches it on disk keyed by
precision, lattices and loop parameters, so later runs of the same workload
start from the tuned shape.  Cache: $WLG_TUNE_CACHE or
~/.cache/wloop_b200/contract_tune.json.
"""
from __future__ import annotations

import json
import os
import time
from typing import Dict, List, Optional, Sequence, Tuple

Shape = Tuple[int, int, int, int]  # (G, SB, block, nCB)


def cache_path() -> str:
    p = os.environ.get("WLG_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "wloop_b200", "contract_tune.json")


def _load() -> Dict[str, list]:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(key: str, shape: Shape) -> None:
    d = _load()
    d[key] = list(shape)
    p = cache_path()
    os.makedirs(os.path.dirname(p), exist_ok=True)
    tmp = p + ".tmp"
    with open(tmp, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, p)


def candidates(msl: int, fp64: bool, batched: bool) -> List[Shape]:
    """Shapes worth timing for msl levels."""
    out: List[Shape] = []
    gs = [g for g in (1, 2, 3, 4) if g <= msl]
    if not batched and not fp64 and msl == 6:
        gs.append(6)
    for G in gs:
        if fp64 and G > 3:
            continue
        # SB 0: the fourth-form family (shared-memory reduction; its best
        # member for the precision); 1, 2: third form; batches also try SB 3,
        # the fourth form with its level loops unrolled (FP32, msl 4-6), SB 5,
        # the same with packed two-lane FMA products (FP32, msl 4-6), and
        # SB 4, the fourth form with bulk-copy staging (FP64)
        if G == 6:
            sbs = (1,)
        elif batched:
            sbs = (0, 1, 2) + ((3, 5) if 4 <= msl <= 6 and not fp64 else ()) + ((4,) if fp64 else ())
        else:
            sbs = (0, 1, 2)
        for SB in sbs:
            for block in ((64,) if fp64 else (64, 128)):
                out.append((G, SB, block, 0))
    if not batched and not fp64 and 4 <= msl <= 6:
        # the ninth form (one 32-column chunk per warp, four blocks per SM),
        # marked SB 9; single contexts only, with its own G and block
        out.append(((msl + 1) // 2, 9, 128, 0))
    # the temporal-gauge form (banded Gram product), marked SB 11; it plans
    # its own shapes (a batch runs it for the lattices whose smearing projects)
    out.insert(0, (0, 11, 0, 0))
    return out


def _apply(ctx, shape: Shape, fp64: bool) -> None:
    G, SB, block, nCB = shape
    if SB == 11:
        ctx.set_contract_tuning(11)
        return
    ctx.set_contract_tuning(_form(G, SB, fp64), G, SB if SB <= 2 else 0, nCB, block)


# the timed scopes of one measurement's loop stage (the temporal-gauge form
# runs its line steps and gauge transformation outside the contraction)
LOOP_SCOPES = ("gauge", "lines", "contract", "reduce")


def key_for(precision: str, lattices: Sequence[tuple], parms) -> str:
    lat = ";".join("x".join(str(v) for v in n) for n in lattices)
    return f"{precision}|{lat}|msl{parms.msl}|t{parms.mwlt}|r{parms.mwlr}"


def cached(key: str) -> Optional[Shape]:
    v = _load().get(key)
    return tuple(v) if v else None


def tune_context(ctx, parms, precision: str, reps: int = 1, use_cache: bool = True) -> Shape:
    """Times the contraction of a Context on its current field (the field is
    restored from a snapshot before every run) and applies the best shape."""
    fp64 = precision == "fp64"
    key = key_for(precision, [ctx.n], parms)
    if use_cache and cached(key):
        _apply(ctx, cached(key), fp64)
        return cached(key)
    ctx.snapshot()
    best, best_t = None, float("inf")
    for (G, SB, block, nCB) in candidates(parms.msl, fp64, batched=False):
        _apply(ctx, (G, SB, block, nCB), fp64)
        ctx.restore()
        ctx.measure(parms)  # warm-up
        ctx.reset_kernel_times()
        ctx.set_profiling(True)
        for _ in range(reps):
            ctx.restore()
            ctx.measure(parms)
        t = sum(ctx.kernel_time(s)[0] for s in LOOP_SCOPES) / max(1, reps)
        ctx.set_profiling(False)
        if t < best_t:
            best, best_t = (G, SB, block, nCB), t
    _apply(ctx, best, fp64)
    ctx.restore()
    _store(key, best)
    return best


def tune_batch(batch, reps: int = 1, use_cache: bool = True) -> Shape:
    """Times whole batch runs (one CUDA-graph launch each) per candidate and
    applies the best shape.  The batch's fields are restored from a snapshot
    before every run."""
    lat = [n for n, _, _ in batch.items]
    p0 = batch.items[0][2]
    key = key_for(batch.precision, lat, p0)
    if use_cache and cached(key):
        batch.set_contract_shape(*_as_batch(cached(key)))
        return cached(key)
    msl = max(p.msl for _, _, p in batch.items)
    batch.snapshot()
    best, best_t = None, float("inf")
    for shape in candidates(msl, batch.precision == "fp64", batched=True):
        batch.set_contract_shape(*_as_batch(shape))
        batch.restore()
        batch.run()  # builds and captures the graph
        t = 0.0
        for _ in range(reps):
            batch.restore()
            batch.run()
            t += batch.stats()[0]
        t /= reps
        if t < best_t:
            best, best_t = shape, t
    batch.set_contract_shape(*_as_batch(best))
    batch.restore()
    _store(key, best)
    return best


def _form(G: int, SB: int, fp64: bool) -> int:
    """kernel form of a context shape: 11 for SB = 11, 9 for SB = 9, 2 for
    G = 6, 3 for SB = 1 or 2, and for SB = 0 the default carried-line form of
    the precision (7 FP64, 10 mixed)"""
    if SB in (9, 11):
        return SB
    if G > 4:
        return 2
    return (7 if fp64 else 10) if SB == 0 else 3


def _as_batch(shape: Shape):
    G, SB, block, nCB = shape
    if SB == 11:
        return 0, 0, 0, 0  # the default plan: the temporal-gauge form where it applies
    return G, SB, nCB, block


# ---------------------------------------------------------------------------
# shapes of the temporal-gauge form's Gram kernel
# ---------------------------------------------------------------------------
def gram_shapes(prec: str):
    """(occ, ord, bx, stages, cpc) candidates: the kernel variants (one block
    of 256, two of 192 or one of 384 threads per SM; dot-product chains or
    one component at a time), start slices per block and pipeline depth;
    cpc 0 = the plan's."""
    bxs = (32, 22, 16) if prec == "mixed" else (0, 16, 8)
    return [(o, r, bx, st, 0) for o in (1, 2, 3) for r in (1, 2) for bx in bxs for st in (0, 2)]


def gram_sweep(ctx, parms, prec: str, shapes=None, reps: int = 2):
    """Times the Gram kernel of ctx's current field for every shape (the field
    is restored from a snapshot before each run); yields one record per
    distinct plan with its launch time and whether the Wilson loops equal
    those of the first plan bit for bit."""
    import numpy as np
    ctx.snapshot()
    ref, seen = None, set()
    for (o, r, bx, st, cpc) in shapes or gram_shapes(prec):
        ctx.set_gram_tuning(o, r, bx, st, cpc)
        try:
            shape = ctx.gram_shape(parms.msl, parms.mwlt)
        except Exception:
            continue  # no kernel of this occupancy for this precision and msl
        key = tuple(sorted(shape.items()))
        if key in seen:
            continue
        seen.add(key)
        ctx.restore()
        wl = ctx.measure(parms)
        if ref is None:
            ref = wl
        ctx.reset_kernel_times()
        ctx.set_profiling(True)
        for _ in range(reps):
            ctx.restore()
            ctx.measure(parms)
        cm, cn = ctx.kernel_time("contract")
        lm, ln = ctx.kernel_time("lines")
        ctx.set_profiling(False)
        yield {"prec": prec, **shape, "gram_ms": cm / max(1, cn), "lines_ms": lm / max(1, ln),
               "max_diff_vs_first": float(np.abs(wl - ref).max())}
    ctx.set_gram_tuning()
    ctx.restore()


def _main():
    import argparse
    ap = argparse.ArgumentParser(description="shape sweeps of the contraction kernels")
    ap.add_argument("--gram-sweep", action="store_true",
                    help="time every Gram kernel shape on the c3 workload (32^3x64)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--cpc", default="", help="comma-separated extra chunk counts per block")
    args = ap.parse_args()
    if not args.gram_sweep:
        ap.error("nothing to do (--gram-sweep)")
    from .api import Context
    from .workloads import C3
    w = C3
    shapes = gram_shapes(args.precision)
    shapes += [(1, 1, 32 if args.precision == "mixed" else 0, 0, int(c))
               for c in args.cpc.split(",") if c]
    with Context(w.n, w.bc, args.precision) as c:
        c.generate(w.seed, w.eps)
        for rec in gram_sweep(c, w.parms, args.precision, shapes):
            print(json.dumps(rec), flush=True)


if __name__ == "__main__":
    _main()
