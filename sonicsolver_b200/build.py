"""Builds the sm_100a library ``sonicsolver_b200/libsonicsolver_b200.so`` in tree.

``python -m sonicsolver_b200.build`` (or ``build()``) compiles every CUDA
translation unit under ``csrc/`` with nvcc for ``sm_100a`` only and links one
shared library exporting the C ABI of ``include/sonicsolver_b200.h``.  Objects
are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libsonicsolver_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
           "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    nvcc = _nvcc()
    headers = _headers()
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if force or _stale(obj, [src] + headers):
            jobs.append([nvcc, *ARCH, *NVFLAGS, "-c", src, "-o", obj])

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    if force or jobs or _stale(LIB, objs):
        run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", LIB, *objs])
    build_host(verbose=verbose, force=force)
    return LIB


HOST = os.path.join(HERE, "host")
RUNNER = os.path.join(HERE, "sfg_run")


def build_host(verbose: bool = False, force: bool = False) -> str:
    """The C++17 host side (case reader, mesh generator, provider catalogs,
    plan, .vts writer) linked into the ``sfg_run`` driver against the library
    (rpath $ORIGIN).  Multiply-adds are not contracted, so the generated
    coordinates and metrics round as the reference's do."""
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    deps = srcs + sorted(glob.glob(os.path.join(HOST, "*.hpp"))) + [os.path.join(ROOT, "include", "sonicsolver_b200.h"), LIB]
    if not (force or _stale(RUNNER, deps)):
        return RUNNER
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-Wextra", "-o", RUNNER, *srcs, "-L", HERE, "-lsonicsolver_b200",
           "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return RUNNER


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
