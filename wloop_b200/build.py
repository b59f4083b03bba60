"""Builds libwloop_b200.so in-tree for sm_100a.

Usage: python wloop_b200/build.py [--force]   (a plain script: importing the
package itself would load the library being built)

Every .cu file is compiled by nvcc with -gencode arch=compute_100a,code=sm_100a;
gen_dev.cu is compiled with --fmad=false and gen_host.cpp with
-ffp-contract=off so the device and host field generators write identical
bytes.  The shared library is written to wloop_b200/_lib/.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libwloop_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
# The image's default CC wrapper lacks libgomp; the system compiler has it.
HOST_CXX = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-ccbin", HOST_CXX,
           "--expt-relaxed-constexpr", "-Xptxas", "-warn-spills"] + ARCH

CU_SOURCES = ["ctx.cu", "smear.cu", "loops.cu", "layout.cu", "gen_dev.cu", "batch.cu", "noalloc.cu", "symm.cu", "gram.cu"]
CXX_SOURCES = ["gen_host.cpp", "legacy.cpp", "serve.cpp", "datfile.cpp", "cnfg.cpp"]


def _sources_present():
    cu = [s for s in CU_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    cx = [s for s in CXX_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    return cu, cx


def _deps():
    files = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                files.append(os.path.join(d, f))
    return files


def _stale(obj, src, deps):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    deps = _deps()
    cu, cx = _sources_present()
    jobs = []
    objs = []
    for s in cu:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        extra = ["--fmad=false"] if s == "gen_dev.cu" else []
        if force or _stale(obj, src, deps):
            jobs.append([NVCC] + NVFLAGS + extra + ["-I", os.path.join(ROOT, "include"),
                                                    "-c", src, "-o", obj])
    for s in cx:
        src = os.path.join(CSRC, s)
        obj = os.path.join(BUILD, s + ".o")
        objs.append(obj)
        flags = ["-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall"]
        if s == "gen_host.cpp":
            flags += ["-ffp-contract=off"]
        if force or _stale(obj, src, deps):
            jobs.append([HOST_CXX] + flags + ["-I", "/usr/local/cuda/include",
                                              "-I", os.path.join(ROOT, "include"),
                                              "-c", src, "-o", obj])
    if jobs:
        with ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            outs = list(ex.map(_run, jobs))
        if verbose:
            for o in outs:
                if o.strip():
                    print(o)
    if force or jobs or not os.path.exists(LIB) or any(
            os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-ccbin", HOST_CXX, "-o", LIB] + objs +
             ["-Xcompiler", "-fopenmp", "-lgomp", "-lpthread"])
    return LIB


def clean():
    shutil.rmtree(BUILD, ignore_errors=True)
    shutil.rmtree(LIBDIR, ignore_errors=True)


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose="-v" in sys.argv))
