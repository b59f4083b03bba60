"""Measurement runs over a list of configurations, as main/ms10.c does them.

ms10 (main/ms10.c:687-760) visits the configurations first, first+step, ...,
last; for each it HYP-smears the gauge field with alpha_action and computes
the Wilson-loop matrices (set_data, ms10.c:633-646), then appends one record
to its .dat file (save_data, ms10.c:649-659).  `run` does the same on the GPU
through the C ABI and writes ms10's files under ms10's names
(ms10.c:254-256): <name>.ms10.dat (head and records through wlg_dat_* of
libwloop_b200.so), <name>.ms10.par (the boundary-condition record, then the
wloop record, in the order ms10 writes them, ms10.c:290-313) and a log
<name>.ms10.log.  The log adds, per configuration, the average plaquette
after the HYP smearing and after every smearing level (lnk_plaq_sum,
lnkplaq.c:117-128, over the number of plaquettes), a diagnostic ms10 itself
does not print (its print_log is commented out, ms10.c:722).

Several processes (one per GPU, launched by torchrun) share a run as
replicas: rank r measures every world-th configuration into its own file
<name>.ms10.r<rank>.dat, and `merge` interleaves those into the single
<name>.ms10.dat ordered by configuration number that one process would have
written.  No device data crosses ranks.

Configurations come from ms10's exported files <cnfg_dir>/<name>n<nc>
(imported into the context with the stored plaquette checked, as openQCD's
import_cnfg does), from a callable nc -> host field (complex128, shape
(V, 4, 3, 3), su3_dble layout), or, without either, are synthetic fields
generated on the device with seed nc.
"""
from __future__ import annotations

import ctypes as C
import os
import time
from dataclasses import dataclass
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np

from ._native import WlgError, dptr, iptr, lib
from .api import Context, WloopParms, plaquette_count
from .replicas import Replicas, config_numbers, shard


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise WlgError(f"{what}: {lib.wlg_dat_error().decode(errors='replace')}")


def _b(path: str) -> bytes:
    return os.fsencode(path)


# ---------------------------------------------------------------------------
# .dat and .par files
# ---------------------------------------------------------------------------
def dat_head(p: WloopParms, n0: int) -> List[int]:
    """[wls, msl, mwlt, mwlr, tmax] of a run (ms10.c:86-105)."""
    h = (C.c_int * 5)()
    cp = p.to_c()
    _check(lib.wlg_dat_head(C.byref(cp), n0, h), "dat_head")
    return list(h)


def write_head(path: str, head: Sequence[int]) -> None:
    _check(lib.wlg_dat_write_head(_b(path), (C.c_int * 5)(*head)), "write_file_head")


def check_head(path: str, head: Sequence[int]) -> None:
    _check(lib.wlg_dat_check_head(_b(path), (C.c_int * 5)(*head)), "check_file_head")


def append(path: str, nc: int, wl: np.ndarray) -> None:
    wl = np.ascontiguousarray(wl, dtype=np.float64)
    _check(lib.wlg_dat_append(_b(path), int(nc), dptr(wl), wl.size), "write_data")


def count(path: str) -> Tuple[List[int], int]:
    """(head, number of complete records)."""
    h = (C.c_int * 5)()
    n = lib.wlg_dat_count(_b(path), h)
    if n < 0:
        _check(-1, "read_data")
    return list(h), int(n)


def read(path: str) -> Tuple[List[int], np.ndarray, np.ndarray]:
    """(head, nc of every record, wl_mat of every record as (records, wls))."""
    head, n = count(path)
    wls = head[0]
    ncs = np.empty(n, dtype=np.int32)
    wl = np.empty((n, wls), dtype=np.float64)
    nc = C.c_int()
    for r in range(n):
        _check(lib.wlg_dat_read(_b(path), r, C.byref(nc), dptr(wl[r]), wls), "read_data")
        ncs[r] = nc.value
    return head, ncs, wl


def merge(parts: Sequence[str], out: str) -> int:
    """Interleaves per-replica .dat files into one, ordered by configuration
    number (stable for repeated numbers).  All parts must share one head.
    Returns the number of records written."""
    head = None
    recs = []
    for i, path in enumerate(parts):
        h, ncs, wl = read(path)
        if head is None:
            head = h
        elif h != head:
            raise WlgError(f"merge: {path} has head {h}, expected {head}")
        recs.extend((int(nc), i, r, wl[r]) for r, nc in enumerate(ncs))
    if head is None:
        raise WlgError("merge: no input files")
    recs.sort(key=lambda x: (x[0], x[1], x[2]))
    write_head(out, head)
    for nc, _, _, w in recs:
        append(out, nc, w)
    return len(recs)


BC_RECORD_BYTES = 4 + 8 * 10


def write_par(path: str, p: WloopParms, bc: Optional[int] = None) -> None:
    """Appends the .par records: with bc given, the boundary-condition record
    first (write_bc_parms, ms10.c:295), then the wloop record
    (write_wloop_parms, wloop_parms.c:343-382)."""
    if bc is not None:
        _check(lib.wlg_par_write_bc(_b(path), int(bc)), "write_bc_parms")
    cp = p.to_c()
    _check(lib.wlg_par_write_wloop(_b(path), C.byref(cp)), "write_wloop_parms")


def check_par(path: str, p: WloopParms, offset: int = 0, bc: Optional[int] = None) -> None:
    """Compares a .par file with the run's parameters: with bc given, the
    boundary-condition record at `offset`, then the wloop record after it."""
    if bc is not None:
        _check(lib.wlg_par_check_bc(_b(path), offset, int(bc)), "check_bc_parms")
        offset += BC_RECORD_BYTES
    cp = p.to_c()
    _check(lib.wlg_par_check_wloop(_b(path), offset, C.byref(cp)), "check_wloop_parms")


# ---------------------------------------------------------------------------
# configurations in openQCD's exported format
# ---------------------------------------------------------------------------
def _cnfg_check(rc: int, what: str) -> None:
    if rc != 0:
        raise WlgError(f"{what}: {lib.wlg_cnfg_error().decode(errors='replace')}")


def cnfg_head(path: str) -> Tuple[Tuple[int, int, int, int], float]:
    """(lattice extents, stored average plaquette) of an exported file."""
    n = (C.c_int * 4)()
    plaq = C.c_double()
    _cnfg_check(lib.wlg_cnfg_read_head(_b(path), n, C.byref(plaq)), "import_cnfg")
    return tuple(n), plaq.value


def import_cnfg(path: str, n=None) -> np.ndarray:
    """The field of an exported configuration as complex128 (V, 4, 3, 3),
    lexicographic sites (the layout Context.upload takes)."""
    if n is None:
        n, _ = cnfg_head(path)
    vol = int(np.prod(n))
    u = np.empty((vol, 4, 3, 3), dtype=np.complex128)
    _cnfg_check(lib.wlg_cnfg_import(_b(path), (C.c_int * 4)(*n), dptr(u.view(np.float64)), None),
                "import_cnfg")
    return u


def export_cnfg(path: str, u: np.ndarray, n, plaq: float) -> None:
    """Writes u (V, 4, 3, 3) in the exported format with the given plaquette
    value in the head."""
    u = np.ascontiguousarray(u, dtype=np.complex128)
    _cnfg_check(lib.wlg_cnfg_export(_b(path), (C.c_int * 4)(*n), dptr(u.view(np.float64)),
                                    float(plaq)), "export_cnfg")


def cnfg_source(cnfg_dir: str, name: str, n) -> Callable[[int], np.ndarray]:
    """nc -> field of <cnfg_dir>/<name>n<nc>, ms10's exported-file naming
    (main/ms10.c:716)."""
    def source(nc: int) -> np.ndarray:
        return import_cnfg(os.path.join(cnfg_dir, f"{name}n{nc}"), tuple(n))
    return source


# ---------------------------------------------------------------------------
# runs
# ---------------------------------------------------------------------------
@dataclass
class Run:
    """One measurement run (the [Run name], [Configurations] and [Wloop]
    sections of ms10's input file, plus the lattice)."""
    name: str
    n: Tuple[int, int, int, int]
    bc: int
    parms: WloopParms
    first: int
    last: int
    step: int = 1
    precision: str = "mixed"
    eps: float = 0.2  # synthetic fields only

    @property
    def configs(self) -> List[int]:
        return config_numbers(self.first, self.last, self.step)


def dat_path(out_dir: str, name: str, rank: int = 0, world: int = 1) -> str:
    if world == 1:
        return os.path.join(out_dir, f"{name}.ms10.dat")
    return os.path.join(out_dir, f"{name}.ms10.r{rank}.dat")


def par_path(out_dir: str, name: str) -> str:
    return os.path.join(out_dir, f"{name}.ms10.par")


def log_path(out_dir: str, name: str) -> str:
    return os.path.join(out_dir, f"{name}.ms10.log")


def end_path(out_dir: str, name: str) -> str:
    """ms10's end flag (ms10.c:662-680): a file of this name stops the run
    after the configuration in progress."""
    return os.path.join(out_dir, f"{name}.ms10.end")


def _equally_spaced(ncs: Sequence[int], what: str) -> Tuple[int, int, int]:
    """(first, last, step) of a list of configuration numbers; they must be
    equally spaced (check_old_log / check_old_dat, ms10.c:374-487)."""
    if not ncs:
        raise WlgError(f"{what}: No data records found")
    step = ncs[1] - ncs[0] if len(ncs) > 1 else 0
    if any(b - a != step for a, b in zip(ncs, ncs[1:])):
        raise WlgError(f"{what}: Configuration numbers are not equally spaced")
    return ncs[0], ncs[-1], step


def check_continuation(r: Run, out_dir: str) -> int:
    """ms10's continuation checks (-a, ms10.c:490-526): the old log and .dat
    report the same equally spaced configurations, the .dat head and the .par
    records (bc, then wloop) are this run's, and the run continues the old
    range at last + step.  Returns the number of records already there."""
    logf, dat, par = log_path(out_dir, r.name), dat_path(out_dir, r.name), par_path(out_dir, r.name)
    for p in (logf, dat, par):
        if not os.path.exists(p):
            raise WlgError(f"check_files: continuation run: {p} does not exist")
    done = []
    with open(logf) as f:
        for ln in f:
            if ln.startswith("Configuration no ") and "fully processed" in ln:
                done.append(int(ln.split()[2]))
    fst, lst, stp = _equally_spaced(done, "check_old_log")
    check_head(dat, dat_head(r.parms, r.n[0]))
    _, ncs, _ = read(dat)
    if (fst, lst, stp) != _equally_spaced([int(x) for x in ncs], "check_old_dat"):
        raise WlgError("check_old_dat: Configuration range is not as reported in the log file")
    check_par(par, r.parms, bc=r.bc)
    if fst != lst and stp != r.step:
        raise WlgError("check_files: Continuation run: "
                       "Previous run had a different configuration separation")
    if r.first != lst + r.step:
        raise WlgError("check_files: Continuation run: "
                       "Configuration range does not continue the previous one")
    return len(ncs)


def _device_measure(run: Run, source, device: int, cnfg_dir: Optional[str] = None):
    """nc -> (wl_mat, average plaquette after HYP, average plaquette of every
    level): hyp_links(alpha_action) then wloop_sum, as Context.measure."""
    ctx = Context(run.n, run.bc, run.precision, device=device)
    p = run.parms
    nplaq = plaquette_count(run.n, run.bc)

    def measure(nc: int):
        if cnfg_dir is not None:
            ctx.import_cnfg(os.path.join(cnfg_dir, f"{run.name}n{nc}"))
        elif source is None:
            ctx.generate(nc, run.eps)
        else:
            ctx.upload(source(nc))
        ctx.hyp_links(*p.alpha_action, p.proj, p.proj_iter)
        plaq_hyp = ctx.lnk_plaq_sum() / nplaq
        wl, pl = ctx.wloop_sum(p, plaq=True)
        return wl, plaq_hyp, pl / nplaq

    return ctx, measure


def run(r: Run, out_dir: str, replicas: Optional[Replicas] = None,
        source: Optional[Callable[[int], np.ndarray]] = None,
        measure: Optional[Callable[[int], np.ndarray]] = None,
        log: Optional[Callable[[str], None]] = None, cnfg_dir: Optional[str] = None,
        continue_run: bool = False, backup: bool = True) -> dict:
    """Measures this rank's share of the run's configurations and appends one
    record per configuration to its .dat file.  `measure` (nc -> wl_mat)
    replaces the device measurement; by default a Context on this rank's
    local GPU runs HYP(alpha_action) + wloop_sum on each configuration, on
    the exported file <cnfg_dir>/<name>n<nc> when cnfg_dir is given.
    Every rank writes its lines to <name>.ms10.log (rank r > 0 to
    <name>.ms10.r<rank>.log) and to `log`.  With several replicas, rank 0
    merges the per-rank files into <name>.ms10.dat after all ranks have
    finished.

    As ms10 (ms10.c:490-526, 662-680, 737-738): a new run refuses to
    overwrite an old <name>.ms10.log or .ms10.dat; continue_run=True continues an
    old run of one process (check_continuation) and adds its records and log
    lines to the old files; a file <name>.ms10.end stops a one-process run
    after the configuration in progress (the file is removed); with backup
    the log and .dat are copied to <file>~ after every configuration."""
    import shutil
    rank = replicas.rank if replicas else 0
    world = replicas.world if replicas else 1
    local = replicas.device if replicas else 0
    os.makedirs(out_dir, exist_ok=True)
    head = dat_head(r.parms, r.n[0])
    path = dat_path(out_dir, r.name, rank, world)
    if continue_run:
        if world > 1:
            raise WlgError("check_files: a continuation run has one process")
        check_continuation(r, out_dir)
    else:
        if rank == 0 and any(os.path.exists(p) for p in (log_path(out_dir, r.name),
                                                         dat_path(out_dir, r.name))):
            raise WlgError("check_files: Attempt to overwrite old *.log or *.dat file")
        write_head(path, head)
        if rank == 0:
            par = par_path(out_dir, r.name)
            if os.path.exists(par):
                os.remove(par)
            write_par(par, r.parms, r.bc)
    logfile = log_path(out_dir, r.name) if rank == 0 else \
        os.path.join(out_dir, f"{r.name}.ms10.r{rank}.log")
    flog = open(logfile, "a" if continue_run else "w")

    def say(line: str) -> None:
        flog.write(line + "\n")
        flog.flush()
        if log:
            log(line)

    mine = shard(r.configs, rank, world)
    ctx = None
    if measure is None:
        ctx, measure = _device_measure(r, source, local, cnfg_dir)
    seconds, processed = [], []
    cum = np.cumsum(r.parms.nss[:r.parms.msl])
    try:
        for nc in mine:
            t0 = time.perf_counter()
            say(f"Configuration no {nc}")
            res = measure(nc)
            wl = res[0] if isinstance(res, tuple) else res
            if wl.size != head[0]:
                raise WlgError(f"measurement of configuration {nc} has {wl.size} entries, "
                               f"expected {head[0]}")
            append(path, nc, wl)
            processed.append(nc)
            seconds.append(time.perf_counter() - t0)
            if isinstance(res, tuple):
                say(f"Average plaquette after HYP smearing = {res[1]:.15e}")
                for sl, v in enumerate(res[2]):
                    say(f"Average plaquette at smearing level {sl} ({int(cum[sl])} sweeps) = "
                        f"{v:.15e}")
            say(f"Configuration no {nc} fully processed in {seconds[-1]:.2e} sec "
                f"(average = {sum(seconds) / len(seconds):.2e} sec)")
            if backup:
                shutil.copyfile(logfile, logfile + "~")
                shutil.copyfile(path, path + "~")
            endf = end_path(out_dir, r.name)
            if world == 1 and os.path.exists(endf):
                os.remove(endf)
                say("End flag set, run stopped")
                break
    finally:
        flog.close()
        if ctx is not None:
            ctx.close()
    out = {"rank": rank, "world": world, "path": path, "configs": processed, "seconds": seconds,
           "log": logfile}
    if world > 1:
        replicas.barrier()
        if rank == 0:
            parts = [dat_path(out_dir, r.name, k, world) for k in range(world)]
            # a rank that failed leaves fewer records than its share: no merge
            for k, part in enumerate(parts):
                want = len(shard(r.configs, k, world))
                have = count(part)[1]
                if have != want:
                    raise WlgError(f"merge: rank {k} wrote {have} of its {want} records "
                                   f"({part}); the merged file is not written")
            out["merged"] = dat_path(out_dir, r.name)
            out["records"] = merge(parts, out["merged"])
        replicas.barrier()
    return out


def main(argv=None) -> int:
    """Command line: python -m wloop_b200.measure --name run1 --lattice 64x32x32x32 ...
    (under torchrun for several GPUs)."""
    import argparse
    from .api import APE, HYP
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--name", required=True)
    ap.add_argument("--out", default=".")
    ap.add_argument("--lattice", required=True, help="N0xN1xN2xN3")
    ap.add_argument("--bc", type=int, default=3, help="0 open, 3 periodic")
    ap.add_argument("--first", type=int, default=1)
    ap.add_argument("--last", type=int, default=1)
    ap.add_argument("--step", type=int, default=1)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--eps", type=float, default=0.2)
    ap.add_argument("--cnfg-dir", default=None,
                    help="read <cnfg-dir>/<name>n<nc> in openQCD's exported format instead of "
                         "generating synthetic fields")
    ap.add_argument("--msl", type=int, required=True)
    ap.add_argument("--nss", type=int, nargs="+", required=True)
    ap.add_argument("--mwlt", type=int, required=True)
    ap.add_argument("--mwlr", type=int, required=True)
    ap.add_argument("--op-smear", default="APE", choices=["APE", "HYP"])
    ap.add_argument("--alpha-action", type=float, nargs=3, default=(1.0, 1.0, 0.5))
    ap.add_argument("--alpha", type=float, nargs="+", default=[0.5])
    ap.add_argument("--proj-iter", type=int, default=4)
    ap.add_argument("-a", "--append", action="store_true",
                    help="continue an old run (ms10 -a): check its files and append")
    a = ap.parse_args(argv)
    n = tuple(int(x) for x in a.lattice.split("x"))
    hyp = a.op_smear == "HYP"
    p = WloopParms(a.msl, a.nss, a.mwlt, a.mwlr, HYP if hyp else APE, tuple(a.alpha_action),
                   0.0 if hyp else a.alpha[0], tuple(a.alpha[:2]) if hyp else (0.0, 0.0),
                   a.proj_iter)
    r = Run(a.name, n, a.bc, p, a.first, a.last, a.step, a.precision, a.eps)
    with Replicas() as rep:
        res = run(r, a.out, rep, log=print if rep.rank == 0 else None, cnfg_dir=a.cnfg_dir,
                  continue_run=a.append)
    if res.get("merged"):
        print(f"{res['records']} records in {res['merged']}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
