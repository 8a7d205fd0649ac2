#!/usr/bin/env python3
"""Benchmark of the B200 explicit Euler provider (one JSON line on rank 0).

Workload: 2-D periodic isentropic vortex, 1024^2 cells on [0, 10]^2,
TENO5 characteristic + Rusanov, SSPRK3, CFL 0.4 (the project's headline
configuration).  A step is one full SSPRK3 time step (device CFL reduction +
3 stages) over the whole grid.  Metric: Mcell-steps/s.

  value     -- device throughput with the state resident in HBM, K steps in
               one CUDA graph, timed with CUDA events on the launching stream;
  e2e       -- the same steps through the public C ABI with host buffers:
               every step uploads the state from pinned host memory,
               advances one CFL step and downloads the state;
  roofline  -- dominant sweep kernel: algorithmic HBM bytes per launch over
               its CUDA-event duration vs the measured HBM copy bandwidth,
               with the FP64/FP32 issue roof beside it (the binding one);
  cpu_baseline -- the reference's own operator (oracle/_ref, compiled from
               the sonicSolver sources) on the host cores.

--impl reference times the reference CPU implementation alone.
--gpus N runs N independent replicas (one per rank, weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# algorithmic HBM bytes per node per launch of each sweep (FP64 state, 5 vars)
#   first axis of 2-D/3-D: read q_s, write R                         -> 80
#   last axis (stage update): read q_s, R, q0, write q_out (+K RK4)   -> 160
STATE_BYTES = 40
# algorithmic FLOPs per face (reconstruction + flux), counted from the kernel
# source: projection 12/pt, WENO5 core ~58 + 1 div, TENO5 core ~70 + 3 div
# (the full cut-off; a smooth stencil skips it and does fewer),
# back-projection 24, Rusanov ~60 + 2 div + 2 sqrt, eigen ~30 + rsqrt.
# DRAM bytes (read + write) of one stage-1 launch of the fused 2-D tile kernel
# on the 1024^2 vortex (variant 1: 32 x 15 tiles, variant 2: 22 x 22), from
# one ncu --set full capture per kernel of the same command line with --quick.
PROFILED_DRAM_BYTES = {("tile2d", 1, 1024, "fp32flux"): 42.300e6 + 7.356e6,
                       ("tile2d", 2, 1024, "fp32flux"): 42.036e6 + 4.637e6,
                       ("tile2d", 2, 1024, "fp64"): 42.113e6 + 5.318e6}
FLOPS_PER_FACE = {"weno5": 6 * 12 + 10 * 59 + 24 + 64 + 34, "teno5": 6 * 12 + 10 * 73 + 24 + 64 + 34}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=1024)
    ap.add_argument("--precision", default="fp32flux", choices=["fp32flux", "fp64"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="skip e2e / peaks / baseline (profiling runs)")
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--serve-requests", type=int, default=96)
    ap.add_argument("--serve-rate", type=float, default=8.0, help="Poisson arrivals per second")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--accuracy-t", type=float, default=10.0, help="vortex run length for the L1 check (0: skip)")
    ap.add_argument("--tgv-t", type=float, default=0.25, help="Taylor-Green run length (0: skip)")
    ap.add_argument("--tgv-size", type=int, default=256)
    ap.add_argument("--curv-t", type=float, default=1.0, help="curvilinear vortex run length (0: skip)")
    ap.add_argument("--all-kernels", action="store_true",
                    help="run every kernel family once on inputs larger than L2 (for a profiler launch list)")
    ap.add_argument("--family", default="all",
                    choices=["all", "vortex2d", "channel", "tube1d", "sod", "tgv3d", "curv", "batch"],
                    help="with --all-kernels: one kernel family's workload only (small profiler captures)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------ CPU legs

def _cpu_worker(args):
    """Reference-operator SSPRK3 steps on one slab of the vortex grid, rows
    y0 .. y0 + ny - 1 (runs in a spawned process)."""
    native, nx, ny, y0, steps, recipe_scheme = args
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle")]
    import numpy as np
    import pyoracle as po
    from sonicsolver_b200 import cases
    L = 10.0
    h = L / 1024
    x = np.arange(nx) * h
    y = (np.arange(ny) + y0) * h
    X, Y = np.meshgrid(x, y, indexing="xy")
    rho, u, v, p = cases.vortex_fields(X, Y, 0.0, L, 5.0, 1.4)
    q = cases.conserved(rho, u, v, 0.0, p)[None]
    spec = po.GridSpec(dim=2, n=(nx, ny, 1), ng=3, h=(h, h, 1.0), bc_lo=(1, 1, 0), bc_hi=(1, 1, 0))
    Q = spec.empty()
    spec.interior(Q)[...] = q
    po.fill_ghosts(spec, Q)
    if native is None:
        t0 = time.perf_counter()
        st = po.Stepper(spec, recipe_scheme, po.RUSANOV, po.SSPRK3)
        for _ in range(steps):
            st.step(Q, po.dt(spec, Q, 0.4))
        return time.perf_counter() - t0
    rc = po.RefCase(spec, recipe_scheme, po.RUSANOV, native=True)
    t0 = time.perf_counter()
    for _ in range(steps):
        rc.step(po.SSPRK3, Q, rc.dt(Q, 0.4))
    return time.perf_counter() - t0


def host_cores() -> int:
    """Cores this process may run on (its CPU affinity), not the machine's."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline(procs=None, nx=1024, rows=1024, steps=3, samples=1, warmup=0):
    """The reference's own operator (oracle/_ref native build for this host's
    CPU target) on the whole 1024^2 vortex grid split into one row slab per
    core of this process's affinity set, as its MPI decomposition runs it
    (the reference is single-threaded per rank); falls back to the oracle
    port.  Each slab is periodic on its own: the halo exchange a decomposed
    run adds is not timed, so the rate is an upper bound for the reference.
    Each sample: every process times `steps` SSPRK3 steps of its slab; the
    sample's rate is the grid's cell-steps over the slowest process's time.
    Reports the median sample."""
    import multiprocessing as mp
    sys.path[:0] = [os.path.join(ROOT, "oracle")]
    import pyoracle as po
    native = True if po.ref_lib(native=True) is not None else None
    kind = "reference" if native else "port"
    flags = po.ref_native_build()[1] if native else "the C oracle port, -O2"
    procs = procs or max(1, min(host_cores(), 64))
    procs = min(procs, rows // 8)          # slabs of at least 8 rows
    share, extra = divmod(rows, procs)
    slabs, y0 = [], 0
    for k in range(procs):
        ny = share + (1 if k < extra else 0)
        slabs.append((native, nx, ny, y0, steps, po.TENO5))
        y0 += ny
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    rates = []
    with ctx.Pool(procs) as pool:
        for k in range(warmup + samples):
            walls = pool.map(_cpu_worker, slabs)
            if k >= warmup:
                rates.append(nx * rows * steps / max(walls) / 1e6)
    total = time.perf_counter() - t0
    value = statistics.median(rates)
    return {"value": value, "unit": "Mcell-steps/s", "cores": procs, "kind": kind,
            "sample": f"{steps} SSPRK3 steps of the whole {nx}x{rows} vortex grid as {procs} row slabs, one "
                      f"process each (each slab periodic on its own: no halo exchange timed), TENO5+Rusanov, "
                      f"reference operator compiled {flags}; median of {len(rates)} sample(s)",
            "per_core": value / procs, "samples": [round(r, 4) for r in rates], "wall_s": round(total, 2)}


# ------------------------------------------------------------------ GPU legs

def run_ours(args, rank, world):
    import numpy as np
    import torch
    from sonicsolver_b200 import capi, cases

    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream()
    prec = capi.PREC_FP32_FLUX if args.precision == "fp32flux" else capi.PREC_FP64
    case = cases.isentropic_vortex(args.size)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        s = case.solver(precision=prec, stream=ctypes_stream(stream))
    from sonicsolver_b200 import autotune
    tuned = autotune.tune_solver(s, "teno5Rusanov", prec)
    K, W = args.steps, args.warmup
    # warm-up (untimed): builds and caches the K-step graph shape too
    s.advance(1e30, max_steps=W, graph_steps=K)
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        st, _ = s.advance(1e30, max_steps=K, graph_steps=K)
        torch.cuda.synchronize()
    barrier(world)
    ms = st.device_ms
    ms_max = allreduce_max(ms, world)
    cells = case.cells
    value = whole_job_rate(cells * K, ms_max, world) / 1e6

    out = {"metric": "Mcell-steps/s", "value": round(value, 2), "unit": "Mcell-steps/s", "n_gpus": world,
           "steps": K, "warmup": W, "ms_per_step": round(ms_max / K, 4), "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None,
           "dtype": "fp32 flux / fp64 state" if prec else "fp64",
           "data": "synthetic (analytic isentropic vortex initial condition)",
           "config": {"workload": "isentropic_vortex_2d", "cells": f"{args.size}x{args.size}", "domain": "[0,10]^2",
                      "recipe": "teno5Rusanov", "time": "SSPRK3", "cfl": 0.4, "precision": args.precision,
                      "parallelism": f"replicas x{world}", "graph_steps": K, "kernel_variant": s.variant,
                      "autotune_ms_per_stage": tuned.get("ms_per_stage"),
                      "l2": "inputs larger than L2 (4 x 42 MB state arrays touched per stage)"},
           "clocks": clk.summary(), "gpu_launches": None}
    dim = case.dim
    launches_per_step = 2 + 3 * (1 if (dim == 2 and s.variant > 0) else dim) + 1  # dt, finalize, stages, commit
    out["gpu_launches"] = launches_per_step * (K + 0)
    if args.quick:
        s.close()
        return out
    s2 = None
    if rank == 0:
        s2 = rank0_comparisons(args, out, s, case, prec, stream, K, W)
    barrier(world)

    # ---- e2e through the C ABI with pinned host buffers, every step, on
    # every rank (replicas); the slowest rank's time counts
    E = args.e2e_steps
    host = torch.empty(case.q.size, dtype=torch.float64, pin_memory=True).numpy()
    host[:] = case.q.ravel()
    t_sim = 0.0
    with torch.cuda.stream(stream):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.upload(host, t_sim)
        s.step()
        s.download(out=host)
        torch.cuda.synchronize()
    barrier(world)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(E):
            s.upload(host, t_sim)      # H2D of the step's input state
            s.step()                   # CFL step (device dt + 3 stages)
            s.download(out=host)       # D2H of the step's result state
        ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    e2e_ms = allreduce_max(ev0.elapsed_time(ev1), world)
    out["e2e"] = {"value": round(whole_job_rate(cells * E, e2e_ms, world) / 1e6, 2), "unit": "Mcell-steps/s",
                  "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(host.nbytes),
                  "steps": E, "path": "sfg_upload(pinned) + sfg_step + sfg_download per step"}
    out["gpu_launches"] += E * (launches_per_step + 2)
    s.close()
    if s2 is not None:
        # the other precision's e2e on the same path (rank 0): the FP64 e2e
        # is the end-to-end figure at the reference's own precision
        with torch.cuda.stream(stream):
            host[:] = case.q.ravel()
            s2.upload(host, t_sim)
            s2.step()
            s2.download(out=host)
            torch.cuda.synchronize()
            ev0.record(stream)
            for _ in range(E):
                s2.upload(host, t_sim)
                s2.step()
                s2.download(out=host)
            ev1.record(stream)
        torch.cuda.synchronize()
        key = "e2e_fp64" if prec else "e2e_fp32flux"
        out[key] = {"value": round(cells * E / (ev0.elapsed_time(ev1) * 1e-3) / 1e6, 2), "unit": "Mcell-steps/s",
                    "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(host.nbytes), "steps": E,
                    "path": "sfg_upload(pinned) + sfg_step + sfg_download per step, rank 0"}
        s2.close()
    if world > 1 or rank != 0:
        return out   # the other workloads are measured by the one-GPU run
    if args.accuracy_t > 0:
        out["accuracy"] = run_accuracy(args)
    out["sod_1d"] = run_sod(args)
    if args.tgv_t > 0:
        out["taylor_green"] = run_taylor_green(args)
    if args.curv_t > 0:
        out["curvilinear"] = run_curvilinear(args)
    if not args.no_batch:
        out["batched"] = {"fp32flux": run_batched(args, capi.PREC_FP32_FLUX), "fp64": run_batched(args, capi.PREC_FP64)}
        out["batched_to_end"] = {
            "fp32flux": run_batched_to_end(args, capi.PREC_FP32_FLUX, out["batched"]["fp32flux"]["tile_variant"]),
            "fp64": run_batched_to_end(args, capi.PREC_FP64, out["batched"]["fp64"]["tile_variant"])}
        e = out["batched_to_end"]
        e["fp32flux_over_fp64"] = round(e["fp32flux"]["value"] / e["fp64"]["value"], 3)
        cap = out["batched"]["fp64"]["value"]
        out["served"] = {"fp32flux": run_served(args, capi.PREC_FP32_FLUX, capacity=cap),
                         "fp64": run_served(args, capi.PREC_FP64, capacity=cap)}
        # capacity of the server for the same request mix: all requests at once
        sat = {"fp32flux": run_served(args, capi.PREC_FP32_FLUX, burst=True),
               "fp64": run_served(args, capi.PREC_FP64, burst=True)}
        sat["fp32flux_over_plain_fp64_single_grid"] = round(
            sat["fp32flux"]["throughput"]["value"] / out["fp64_value"], 3) if out.get("fp64_value") else None
        out["served_saturated"] = sat
    return out


def rank0_comparisons(args, out, s, case, prec, stream, K, W):
    """Rank 0 only (no collectives): the other precision on the same
    workload, and the roofline of the dominant launch.  Returns the
    other-precision solver (closed by the caller)."""
    import numpy as np
    import torch
    from sonicsolver_b200 import capi
    cells, dim = case.cells, case.dim
    # ---- the other precision, same workload (plain FP64 vs mixed)
    other = capi.PREC_FP64 if prec else capi.PREC_FP32_FLUX
    key = "fp64_value" if prec else "fp32flux_value"
    s2 = None
    try:
        with torch.cuda.stream(stream):
            s2 = case.solver(precision=other, stream=ctypes_stream(stream))
        s2.advance(1e30, max_steps=W, graph_steps=K)
        torch.cuda.synchronize()
        st2, _ = s2.advance(1e30, max_steps=K, graph_steps=K)
        out[key] = round(cells * K / (st2.device_ms * 1e-3) / 1e6, 2)
    except capi.SolverError as e:
        out[key] = None
        out[key + "_error"] = str(e)

    # ---- roofline of the dominant launch (a fused stage is timed as 20
    # back-to-back launches in one captured graph, as it runs in a step)
    dt = s.compute_dt()
    ms_axes = s.time_sweeps(dt, stage=0, repeats=20)
    nodes = case.nodes
    hbm, src = measured_peaks()
    dom = int(np.argmax(ms_axes))
    fused = dim == 2 and s.variant > 0
    if fused:
        # one fused launch per stage; the timed launch is stage 1 (read Q^n,
        # write Q1: 80 B per node; stages 2 and 3 also read Q^n: 120 B)
        bytes_node = 2 * STATE_BYTES
    else:
        bytes_node = 2 * STATE_BYTES if (dim > 1 and dom == 0) else 4 * STATE_BYTES
    achieved = bytes_node * nodes / (ms_axes[dom] * 1e-3) / 1e9
    fp_peak = capi.fma_peak_tflops(fp64=(prec == capi.PREC_FP64), seconds=0.5)
    faces = nodes * (dim if fused else 1)  # faces evaluated by one launch
    fl = FLOPS_PER_FACE["teno5"] * faces / (ms_axes[dom] * 1e-3) / 1e12
    traffic = PROFILED_DRAM_BYTES.get(("tile2d", s.variant, args.size, args.precision)) if fused else None
    ms_step = out["ms_per_step"]
    step_gbs = 320 * cells / (ms_step * 1e-3) / 1e9   # SSPRK3, FP64 state: 80 + 120 + 120 B per cell-step
    out["roofline"] = {"bound": "issue", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                       "frac": round(achieved / hbm, 4), "traffic": traffic,
                       "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one stage-1 launch; "
                                       "the output still resident in the write-back L2 at kernel end is not counted",
                       "peak_source": f"{src} (MEASURED_PEAKS.json)",
                       "kernel": ("tile2d fused stage" if fused else f"sweep axis {dom}"),
                       "ms_per_launch": round(ms_axes[dom], 4),
                       "ms_per_launch_timing": ("20 stage-1 launches captured in one CUDA graph, events around "
                                                "the graph" if fused else "launch by launch"),
                       "ms_per_axis": [round(x, 4) for x in ms_axes],
                       "algorithmic_bytes_per_launch": int(bytes_node * nodes),
                       "hbm_step_average": {"achieved": round(step_gbs, 1), "frac": round(step_gbs / hbm, 4),
                                            "bytes_per_cell_step": 320,
                                            "note": "320 B per cell-step (stage 1 80 B, stages 2-3 120 B each) "
                                                    "over the in-graph ms_per_step"},
                       "issue_roof": {"unit": "TFLOP/s", "achieved": round(fl, 2), "fma_peak": round(fp_peak, 2),
                                      "frac": round(fl / fp_peak, 4) if fp_peak else None,
                                      "arith": "fp32" if prec else "fp64",
                                      "flops_per_face": FLOPS_PER_FACE["teno5"],
                                      "peak_source": "measured (sfg_measure_fma_peak: dependent-FMA loop, "
                                                     "this GPU, this run)"},
                       "note": "bound = the binding roof: arithmetic issue (issue_roof), not HBM; achieved / "
                               "peak / frac are the HBM figures on algorithmic bytes of the timed launch"}

    return s2


def run_accuracy(args):
    """Matched-accuracy check on the headline workload: one full period
    (t = 10) of the 1024^2 vortex, TENO5 + Rusanov, SSPRK3, CFL 0.4, in FP64
    and FP32-flux; L1(rho) against the exact solution (the advected initial
    field) and FP32 against FP64 (the FP64 path matches the CPU oracle to
    <= 1e-12 per step in the parity tests; the oracle itself would need days
    on the host for this run), plus the TENO5 cut-off flip rate."""
    import numpy as np
    from sonicsolver_b200 import capi, cases
    case = cases.isentropic_vortex(args.size)
    out = {"t_end": args.accuracy_t, "cells": f"{args.size}x{args.size}"}
    res = {}
    import math

    def sums(a):
        a = a.reshape(-1, 5)
        return [math.fsum(a[:, v]) for v in range(5)], np.abs(a).sum(axis=0)

    tot0, scale = sums(case.q)
    for name, prec in (("fp64", capi.PREC_FP64), ("fp32flux", capi.PREC_FP32_FLUX)):
        s = case.solver(precision=prec)
        d0, f0 = s.teno_flips()
        dev0 = s.totals()
        st, _ = s.advance(args.accuracy_t, graph_steps=64)
        q = s.download().reshape(case.q.shape)
        tot1, _ = sums(q)
        dev1 = s.totals()
        d1, f1 = s.teno_flips()
        ex = cases.vortex_exact(case, st.time)
        res[name] = q
        out[name] = {"steps": int(st.steps), "device_s": round(st.device_ms / 1e3, 3),
                     "l1_rho_vs_exact": float(np.mean(np.abs(q[..., 0] - ex[..., 0]))),
                     "linf_rho_vs_exact": float(np.max(np.abs(q[..., 0] - ex[..., 0]))),
                     # drift of the conserved totals over the run: (sum_t - sum_0) / sum |q_0| per
                     # variable (rho, rho u, rho v, rho w, E), host fsum and sfg_conserved_totals (FP64)
                     "totals_drift": [(a - b) / c if c > 0 else a - b for a, b, c in zip(tot1, tot0, scale)],
                     "totals_drift_device": [(a - b) / abs(b) if b else a - b for a, b in zip(dev1, dev0)]}
        if name == "fp64":
            out["teno_flip_rate"] = {"initial": f0 / max(d0, 1), "final": f1 / max(d1, 1),
                                     "decisions_per_eval": int(d0)}
        s.close()
    out["l1_rho_fp32flux_vs_fp64"] = float(np.mean(np.abs(res["fp32flux"][..., 0] - res["fp64"][..., 0])))
    out["totals_drift_fp32flux_minus_fp64"] = [a - b for a, b in zip(out["fp32flux"]["totals_drift"],
                                                                      out["fp64"]["totals_drift"])]
    out["l1_ratio_fp32flux_over_fp64"] = out["fp32flux"]["l1_rho_vs_exact"] / out["fp64"]["l1_rho_vs_exact"]
    return out


def run_sod(args, repeats=5):
    """Sod shock tube, 1000 cells, WENO5 + Rusanov, SSPRK3, CFL 0.5, t = 0.2,
    FP64: the latency case.  Reports the device time of sfg_advance and the
    wall time of one solve through the C ABI with host buffers (upload +
    advance + download; the solver is created beforehand), median of
    `repeats`, beside the reference operator (oracle/_ref, one host core)
    running the same solve, and the largest relative difference between the
    two final states (the per-step parity bar is in the tests)."""
    import numpy as np
    import torch
    from sonicsolver_b200 import capi, cases
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    case = cases.sod_1d(1000)
    q = np.ascontiguousarray(case.q)
    host = np.empty_like(q)
    walls, devs, steps = [], [], 0
    for r in range(repeats + 1):
        s = case.solver(precision=capi.PREC_FP64)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.upload(q)
        st, _ = s.advance(case.t_end, graph_steps=32)
        s.download(out=host)
        wall = time.perf_counter() - t0
        s.close()
        if r:                                     # the first solve loads modules
            walls.append(wall)
            devs.append(st.device_ms / 1e3)
        steps = int(st.steps)
    # the same solve on the CUDA-graph path (1-D variant 1), for comparison
    # with the whole-run cluster kernel the default variant 2 uses
    graph_devs = []
    for r in range(3):
        s = case.solver(precision=capi.PREC_FP64)
        s.variant = 1
        s.upload(q)
        st1, _ = s.advance(case.t_end, graph_steps=32)
        graph_devs.append(st1.device_ms / 1e3)
        s.close()
    out = {"cells": 1000, "t_end": case.t_end, "steps": steps, "recipe": "weno5Rusanov", "time": "SSPRK3",
           "path": "whole-run cluster kernel (1-D variant 2)",
           "device_s": float(np.median(devs)), "wall_s_capi_host_buffers": float(np.median(walls)),
           "device_s_graph_path": float(np.median(graph_devs[1:]))}
    out["value"] = round(1000 * steps / out["wall_s_capi_host_buffers"] / 1e6, 3)
    out["unit"] = "Mcell-steps/s"
    # L1(rho) against the exact Riemann solution at the final time (nodes
    # x_i = i h); the diaphragm at 0.5
    x = np.arange(case.n[0]) * case.h[0]
    rho_exact = cases.sod_exact(x, case.t_end)[0]
    out["l1_rho_vs_exact"] = float(np.mean(np.abs(host.reshape(-1, 5)[:, 0] - rho_exact)))
    try:
        spec = po.GridSpec(dim=1, n=tuple(case.n), ng=3, h=tuple(case.h), bc_lo=tuple(case.bc_lo),
                           bc_hi=tuple(case.bc_hi), gamma=case.gamma)
        Q = spec.empty()
        spec.interior(Q)[...] = q.reshape(spec.interior(Q).shape)
        po.fill_ghosts(spec, Q)
        rc = po.RefCase(spec, po.WENO5, po.RUSANOV, native=True)
        t0 = time.perf_counter()
        dts, tf = rc.advance(po.SSPRK3, Q, case.t_end, case.cfl)
        ref_s = time.perf_counter() - t0
        ref = np.ascontiguousarray(spec.interior(Q)).reshape(host.shape)
        scale = np.maximum(np.abs(ref).reshape(-1, 5).max(axis=0), 1e-300)
        diff = (np.abs(host - ref).reshape(-1, 5).max(axis=0) / scale)
        out["reference_cpu"] = {"wall_s": ref_s, "steps": int(len(dts)), "cores": 1,
                                "kind": "reference operator, " + po.ref_native_build()[1]}
        out["max_rel_diff_vs_reference"] = float(diff.max())
        out["speedup_wall_vs_reference"] = round(ref_s / out["wall_s_capi_host_buffers"], 2)
    except Exception as e:  # reference library missing on this host
        out["reference_cpu"] = {"unavailable": str(e)}
    return out


def run_taylor_green(args):
    """3-D inviscid Taylor-Green vortex, periodic [0, 2 pi]^3 (256^3 cells by
    default), Mach 0.1, WENO5 + Rusanov, SSPRK3, CFL 0.5, advanced to
    t = args.tgv_t in FP64 and in FP32-flux / FP64-state.  Reports the
    device-timed throughput of each, the kinetic energy KE(t) / KE(0) and the
    FP32-flux kinetic-energy drift relative to the FP64 path (which matches
    the CPU oracle to <= 1e-12 per step in the parity tests)."""
    import numpy as np
    from sonicsolver_b200 import capi, cases
    N = args.tgv_size
    case = cases.taylor_green(N, t_end=args.tgv_t)
    cells = N ** 3
    ke0 = cases.kinetic_energy(case.q)
    out = {"t_end": args.tgv_t, "cells": f"{N}^3", "recipe": "weno5Rusanov", "time": "SSPRK3", "cfl": case.cfl,
           "mach": 0.1, "ke0": ke0}
    res = {}
    from sonicsolver_b200 import autotune
    for name, prec in (("fp64", capi.PREC_FP64), ("fp32flux", capi.PREC_FP32_FLUX)):
        s = case.solver(precision=prec)
        tuned = autotune.tune_solver(s, "weno5Rusanov", prec)   # 0: axis sweeps, 1: z-marching tiles
        s.upload(np.ascontiguousarray(case.q))
        st, _ = s.advance(args.tgv_t, graph_steps=32)
        q = s.download().reshape(case.q.shape)
        ke = cases.kinetic_energy(q)
        res[name] = (q, ke)
        out[name] = {"steps": int(st.steps), "device_s": round(st.device_ms / 1e3, 3),
                     "value": round(cells * st.steps / (st.device_ms * 1e-3) / 1e6, 2), "unit": "Mcell-steps/s",
                     "ke_over_ke0": ke / ke0, "kernel_variant": int(tuned["best"]),
                     "autotune_ms_per_stage": tuned["ms_per_stage"]}
        s.close()
    (q64, ke64), (q32, ke32) = res["fp64"], res["fp32flux"]
    out["ke_drift_fp32flux_vs_fp64"] = (ke32 - ke64) / ke64
    out["ke_change_fp64"] = (ke64 - ke0) / ke0
    out["ke_drift_over_ke_change"] = (ke32 - ke64) / abs(ke64 - ke0) if ke64 != ke0 else None
    out["l1_rho_fp32flux_vs_fp64"] = float(np.mean(np.abs(q32[..., 0] - q64[..., 0])))
    out["fp32flux_over_fp64"] = round(out["fp32flux"]["value"] / out["fp64"]["value"], 3)
    return out


def run_curvilinear(args):
    """The curvilinear path (sfg_set_metrics: per-node metrics, full
    eigenvector faces along each face normal, FP64) on the headline vortex
    moved onto a sheared periodic mesh (cases.wavy_vortex, shear amplitude
    0.3), TENO5 + Rusanov, SSPRK3, CFL 0.4, to t = args.curv_t, in FP64 and
    in FP32-flux / FP64-state: device-timed throughput against the uniform
    FP64 path on the same node count, L1(rho) of each against the exact
    solution at the nodes' physical coordinates, and the time of one stage
    (the fused 2-D tile kernel) with its algorithmic bytes."""
    import numpy as np
    from sonicsolver_b200 import capi, cases
    N = args.size
    out = {"t_end": args.curv_t, "cells": f"{N}x{N}", "mesh": "x = i h + A sin(2 pi j/N), y = j h + A sin(2 pi i/N)",
           "amp": 0.3, "recipe": "teno5Rusanov"}
    runs = (("curvilinear", cases.wavy_vortex(N), capi.PREC_FP64),
            ("curvilinear_fp32flux", cases.wavy_vortex(N), capi.PREC_FP32_FLUX),
            ("uniform", cases.isentropic_vortex(N), capi.PREC_FP64))
    for name, case, prec in runs:
        s = case.solver(precision=prec)
        stage_ms = s.time_sweeps(1e-4, 0, 10)[0]   # one stage (state restored below)
        s.upload(np.ascontiguousarray(case.q))
        st, _ = s.advance(args.curv_t, graph_steps=32)
        q = s.download().reshape(case.q.shape)
        ex = cases.vortex_exact(case, st.time)
        out[name] = {"steps": int(st.steps), "device_s": round(st.device_ms / 1e3, 3),
                     "value": round(N * N * st.steps / (st.device_ms * 1e-3) / 1e6, 2), "unit": "Mcell-steps/s",
                     "l1_rho_vs_exact": float(np.mean(np.abs(q[..., 0] - ex[..., 0]))),
                     "ms_per_stage": None if stage_ms is None else round(float(stage_ms), 4)}
        s.close()
    # algorithmic bytes of one stage-1 launch of the fused 2-D tile kernel per
    # node: the state in (40 B) and out (40 B), the face geometry of two
    # axes (2 x 32 B) and Jac (8 B)
    out["bytes_per_node_stage"] = 40 + 40 + 2 * 32 + 8
    c = out["curvilinear"]
    if c["ms_per_stage"]:
        out["hbm_gbs_per_stage"] = round(out["bytes_per_node_stage"] * N * N / (c["ms_per_stage"] * 1e-3) / 1e9, 1)
    out["curvilinear_over_uniform"] = round(c["value"] / out["uniform"]["value"], 3)
    c32 = out["curvilinear_fp32flux"]
    out["fp32flux_over_fp64"] = round(c32["value"] / c["value"], 3)
    out["l1_ratio_fp32flux_over_fp64"] = c32["l1_rho_vs_exact"] / c["l1_rho_vs_exact"]
    return out


def run_batched(args, precision):
    """Batched shock tubes: 512 seeded instances (half 1-D N in [256, 16384],
    half 2-D side in [64, 512]), WENO5 + Rusanov, SSPRK3, every grid with its
    own CFL step; a bounded number of batch steps timed with CUDA events; a
    1-D and a 2-D instance checked against the plain FP64 path."""
    import torch
    from sonicsolver_b200 import capi, cases
    from sonicsolver_b200 import autotune
    tubes = cases.shock_tube_batch(count=512, seed=2024, t_end=0.15)
    variant = autotune.tune_batch(lambda: capi.Batch(8 << 30, 512, recipe="weno5Rusanov", precision=precision, cfl=0.5),
                                  tubes[::8], "weno5Rusanov", precision)
    b = capi.Batch(8 << 30, 512, recipe="weno5Rusanov", precision=precision, cfl=0.5)
    b.variant = variant
    slots = [b.add(c) for c in tubes]
    steps = args.batch_steps
    b.step(3, graph_steps=16)                     # warm-up (graph capture)
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    before = {s: b.status(s)["steps"] for s in slots}
    t0.record()
    b.step(steps, graph_steps=16)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    cell_steps = sum(c.cells * (b.status(s)["steps"] - before[s]) for c, s in zip(tubes, slots))
    info = b.info()
    # accuracy: a 1-D and a 2-D instance of the batch against the same tube
    # run alone as a plain FP64 single grid over the same steps
    import numpy as np
    l1 = {}
    for dim in (1, 2):
        k = next(i for i, c in enumerate(tubes) if c.dim == dim)
        c, st = tubes[k], b.status(slots[k])
        got = b.download(slots[k]).reshape(c.q.shape)
        alone = c.solver(precision=capi.PREC_FP64)
        alone.advance(c.t_end, max_steps=st["steps"], graph_steps=16)   # same end-time clipping
        ref = alone.download().reshape(c.q.shape)
        alone.close()
        l1[f"{dim}d_instance_{k}"] = float(np.mean(np.abs(got[..., 0] - ref[..., 0])) / np.mean(np.abs(ref[..., 0])))
        if dim == 1:  # the 1-D tube against its exact Riemann solution (unit domain, diaphragm at 0.5)
            x = np.arange(c.n[0]) * c.h[0]
            ex = cases.sod_exact(x, st["time"], c.gamma, c.meta["left"], c.meta["right"])[0]
            l1_exact = {"instance": k, "time": st["time"],
                        "fp_under_test": float(np.mean(np.abs(got.reshape(-1, 5)[:, 0] - ex))),
                        "plain_fp64_alone": float(np.mean(np.abs(ref.reshape(-1, 5)[:, 0] - ex)))}
    b.close()
    return {"value": round(cell_steps / (ms * 1e-3) / 1e6, 2), "unit": "Mcell-steps/s", "batch_steps": steps,
            "instances": len(tubes), "cells_total": int(sum(c.cells for c in tubes)),
            "tiles": info["items"], "ms": round(ms, 2), "tile_variant": variant,
            "note": "default stream events around sfg_batch_step (graph of 16 steps, per-grid dt)",
            "l1_rho_vs_fp64_alone": l1, "l1_rho_vs_exact_1d": l1_exact}


def run_batched_to_end(args, precision, variant):
    """The batched workload run to its end time: all 512 seeded tubes from
    t = 0 to t_end = 0.15, every tube with its own CFL steps, finished tubes
    dropping out of the work list (auto-compaction).  Reports the time to
    solution of the whole batch (CUDA events around the run), the throughput
    including the tail (every cell-step of every tube over that time), and
    how many tubes and work items are live along the way."""
    import numpy as np
    import torch
    from sonicsolver_b200 import capi, cases
    tubes = cases.shock_tube_batch(count=512, seed=2024, t_end=0.15)
    b = capi.Batch(8 << 30, 512, recipe="weno5Rusanov", precision=precision, cfl=0.5)
    b.variant = variant
    slots = [b.add(c) for c in tubes]
    live0 = b.info()["items"]
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    wall0 = time.perf_counter()
    t0.record()
    timeline = []
    calls = 0
    while True:
        active = b.step(64, graph_steps=16)
        calls += 1
        if calls % 8 == 0 or active == 0:
            timeline.append((round(time.perf_counter() - wall0, 3), int(active), int(b.info()["items"])))
        if active == 0:
            break
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    st = [b.status(sl) for sl in slots]
    steps = np.array([x["steps"] for x in st])
    cell_steps = int(sum(c.cells * n for c, n in zip(tubes, steps)))
    reached = [k for k, x in enumerate(st) if abs(x["time"] - 0.15) < 1e-12 and x["flags"] == 0]
    failed = [{"tube": k, "cells": tubes[k].cells, "flags": int(x["flags"]), "steps_done": int(x["steps"]) - 1,
               "time": x["time"]} for k, x in enumerate(st) if x["flags"]]
    b.close()
    keep = np.unique(np.linspace(0, len(timeline) - 1, min(24, len(timeline))).astype(int))
    return {"tubes": len(tubes), "t_end": 0.15, "reached_t_end": len(reached),
            "failed": failed,
            "failed_note": "tubes whose state went invalid (near-vacuum states of the seeded draw): each "
                           "stops with its status bits and the others run on (the reference exits the process "
                           "at that point)",
            "time_to_solution_s": round(ms / 1e3, 3), "cell_steps": cell_steps,
            "value": round(cell_steps / (ms * 1e-3) / 1e6, 2), "unit": "Mcell-steps/s",
            "steps_per_tube": {"min": int(steps.min()), "median": int(np.median(steps)), "max": int(steps.max())},
            "work_items_at_start": int(live0), "tile_variant": variant,
            "timeline": [{"wall_s": timeline[i][0], "running_tubes": timeline[i][1], "work_items": timeline[i][2]}
                         for i in keep],
            "note": "timeline sampled every 512 batch steps (graph launches of 16 steps, 64 per host call)"}


def run_served(args, precision, seed=7, capacity=None, burst=False):
    """Served stream: Poisson arrivals of 2-D solves, a seeded mix of the
    vortex workload's generator (isentropic vortex, TENO5 + Rusanov, CFL 0.4)
    and the batched-tube workload's 2-D generator (slanted shock tubes,
    WENO5 + Rusanov, CFL 0.5), each request with its own recipe and CFL in
    one server; grids 64^2..1024^2, 100..2000 steps, admission by a 60 GB HBM
    budget, continuous batching; latency = finish - submit; the served
    results of the smallest requests against the plain FP64 path.
    `burst`: every request submitted at once (the server saturated), so the
    throughput is the server's capacity for this request mix."""
    import numpy as np
    from sonicsolver_b200 import capi, cases
    rng = np.random.default_rng(seed)
    nreq = args.serve_requests
    reqs = []
    for k in range(nreq):
        side = int(round(np.exp(rng.uniform(np.log(64), np.log(1024)))))
        steps = int(rng.integers(100, 2001))
        if rng.random() < 0.5:
            c = cases.isentropic_vortex(side, recipe="teno5Rusanov", cfl=0.4, t_end=1e9)
        else:
            c = cases.shock_tube_batch(count=2, seed=int(rng.integers(1 << 30)), t_end=1e9, max_2d=side)[1]
        reqs.append((c, steps))
    work = sum(c.cells * s for c, s in reqs)
    srv = capi.Server(60 << 30, 256, recipe="weno5Rusanov", precision=precision, cfl=0.5, graph_steps=8)
    # offered load: 1.2x the plain FP64 path's capacity for this request mix
    rate = args.serve_rate if capacity is None else 1.2 * capacity * 1e6 / (work / nreq)
    gaps = rng.exponential(1.0 / rate, nreq)
    if burst:
        gaps[:] = 0.0
    ids = []
    start = srv.now()
    t_next = start
    for (c, steps), gap in zip(reqs, gaps):
        t_next += gap
        while srv.now() < t_next:
            time.sleep(min(0.002, max(0.0, t_next - srv.now())))
        ids.append(srv.submit(c, max_steps=steps, recipe=c.recipe, cfl=c.cfl))
    srv.drain(600)
    infos = [srv.poll(i) for i in ids]
    end = max(i.finish_s for i in infos)
    lat = np.array([i.finish_s - i.submit_s for i in infos])
    wait = np.array([i.admit_s - i.submit_s for i in infos])
    ok = sum(1 for i in infos if i.state == capi.REQ_DONE)
    failed = [{"request": k, "cells": reqs[k][0].cells, "case": reqs[k][0].name, "flags": int(infos[k].flags),
               "steps_done": int(infos[k].steps)} for k in range(nreq) if infos[k].state == capi.REQ_FAILED]
    # accuracy of served results: the four smallest finished requests rerun
    # alone as plain FP64 single grids over the same steps; L1(rho) of the
    # served state against them, relative to the mean |rho|
    done = sorted((reqs[k][0].cells, k) for k in range(nreq) if infos[k].state == capi.REQ_DONE)[:4]
    l1 = []
    for _, k in done:
        c, steps = reqs[k]
        served_q = srv.fetch(ids[k]).reshape(c.q.shape)
        alone = c.solver(precision=capi.PREC_FP64)
        alone.advance(1e9, max_steps=steps, graph_steps=16)
        ref = alone.download().reshape(c.q.shape)
        alone.close()
        l1.append(float(np.mean(np.abs(served_q[..., 0] - ref[..., 0])) / np.mean(np.abs(ref[..., 0]))))
    # the smallest finished vortex request against the exact advected vortex
    vort = sorted((reqs[k][0].cells, k) for k in range(nreq)
                  if infos[k].state == capi.REQ_DONE and reqs[k][0].name.startswith("isentropic"))
    l1_exact = None
    if vort:
        k = vort[0][1]
        c = reqs[k][0]
        served_q = srv.fetch(ids[k]).reshape(c.q.shape)
        ex = cases.vortex_exact(c, infos[k].time)
        l1_exact = {"request": k, "cells": c.cells, "time": infos[k].time,
                    "l1_rho": float(np.mean(np.abs(served_q[..., 0] - ex[..., 0])))}
    srv.close()
    return {"requests": nreq, "completed": ok, "failed": failed, "arrival_rate_per_s": round(rate, 3),
            "offered_load": ("all requests at t = 0 (saturated)" if burst else
                             "1.2x FP64 batched capacity" if capacity else "fixed rate"),
            "p50_latency_s": round(float(np.percentile(lat, 50)), 4),
            "p99_latency_s": round(float(np.percentile(lat, 99)), 4),
            "p50_queue_wait_s": round(float(np.percentile(wait, 50)), 4),
            "throughput": {"value": round(work / (end - start) / 1e6, 2), "unit": "Mcell-steps/s"},
            "wall_s": round(end - start, 2), "budget_gb": 60,
            "l1_rho_vs_fp64_alone": {"max": max(l1) if l1 else None, "requests": [k for _, k in done],
                                     "note": "relative L1(rho) of the served state against the same request run "
                                             "alone as a plain FP64 single grid"},
            "l1_rho_vs_exact_vortex": l1_exact}


def run_all_kernels(args):
    """One CFL step (or the equivalent launch) of every kernel family of the
    provider, each on a state larger than the 126 MB L2 where the kernel
    streams the state, for a profiler launch list of device time and DRAM
    bytes per kernel (achieved HBM GB/s against the peak).  Timing comes from
    the profiler; this only runs the launches and says what ran."""
    import numpy as np
    from sonicsolver_b200 import capi, cases
    F64, F32 = capi.PREC_FP64, capi.PREC_FP32_FLUX
    ran = []
    fam = args.family

    def want(f):
        return fam in ("all", f)

    def steps(case, label, variants, precisions=(F64, F32)):
        for prec in precisions:
            for v in variants:
                s = case.solver(precision=prec)          # upload (aos_to_soa; geometry when curvilinear)
                s.variant = v
                s.step()                                 # dt, finalize, the stages, commit
                s.close()
                ran.append(f"{label} variant {v} {'fp64' if prec == F64 else 'fp32flux'}: one CFL step")

    # 2-D vortex 2048^2 (168 MB per state copy): axis sweeps, 32 x 15 and 22 x 22 tiles
    if want("vortex2d") or want("channel"):
        vortex = cases.isentropic_vortex(2048)
    if want("vortex2d"):
        steps(vortex, "2-D vortex 2048^2", (0, 1, 2))
        s = vortex.solver()
        s.totals()
        s.teno_flips()
        s.download()
        r = s.residual()
        s.stage_with_residual(0, 1e-4, r)
        s.close()
        ran.append("2-D vortex 2048^2: totals, TENO flip count, download, residual, stage from a given residual")
    if want("channel"):
        # 2-D channel with law ends (fixedValue inflow, zeroGradient outflow)
        lo, hi = (capi.BC_LAW, capi.BC_TRANSMISSIVE, 0), (capi.BC_LAW, capi.BC_TRANSMISSIVE, 0)
        s = capi.Solver(2, vortex.n, vortex.h, lo, hi, recipe="teno5Rusanov", cfl=0.4)
        s.set_boundary_law(0, 0, rho=capi.LAW_FIXED_VALUE, velocity=capi.LAW_FIXED_VALUE, rho_value=1.0,
                           velocity_value=(1.0, 0.0, 0.0))
        s.set_boundary_law(0, 1)
        s.upload(np.ascontiguousarray(vortex.q))
        s.step()
        s.close()
        ran.append("2-D channel 2048^2 with law ends: one CFL step (law fill before each stage)")
    if want("vortex2d") or want("channel"):
        del vortex
    # 1-D tube of 4 M nodes (168 MB): 511-node tiles; Sod 1000 cells: the whole-run cluster kernel
    if want("tube1d"):
        steps(cases.sod_1d((1 << 22) - 1), "1-D tube 4M nodes", (1,))
    if want("sod"):
        sod = cases.sod_1d(1000)
        s = sod.solver()
        s.advance(sod.t_end, max_steps=50)
        s.close()
        ran.append("Sod 1000 cells: 50 steps in one cluster launch")
    # 3-D Taylor-Green 160^3 (164 MB): axis sweeps and z-marching tiles
    if want("tgv3d"):
        steps(cases.taylor_green(160), "3-D Taylor-Green 160^3", (0, 1))
    # curvilinear vortex 1448^2 (84 MB state + 168 MB metrics): face launches and fused tiles
    if want("curv"):
        steps(cases.wavy_vortex(1448), "curvilinear vortex 1448^2", (0, 1))
    # batch: every second tube of the batched workload
    tubes = cases.shock_tube_batch(count=512, seed=2024, t_end=0.15)[::2] if want("batch") else []
    for prec in ((F64, F32) if want("batch") else ()):
        b = capi.Batch(4 << 30, len(tubes), recipe="weno5Rusanov", precision=prec, cfl=0.5)
        for c in tubes:
            b.add(c)
        b.step(2, graph_steps=2)
        b.close()
        ran.append(f"batch of {len(tubes)} tubes ({sum(c.cells for c in tubes)} cells) "
                   f"{'fp64' if prec == F64 else 'fp32flux'}: two batch steps")
    return {"kernels_run": ran}


def ctypes_stream(stream):
    import ctypes
    return ctypes.c_void_p(stream.cuda_stream)


from sonicsolver_b200.replicas import barrier, max_over_ranks as allreduce_max, whole_job_rate  # noqa: E402


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        t0 = time.time()
        # each step a bounded sample: 3 SSPRK3 steps of the whole grid, one row
        # slab per host core
        best = cpu_baseline(steps=3, samples=max(1, min(args.steps, 10)), warmup=min(args.warmup, 1))
        line = {"impl": "reference", "metric": "Mcell-steps/s", "value": round(best["value"], 4),
                "unit": "Mcell-steps/s", "n_gpus": args.gpus, "steps": len(best["samples"]),
                "warmup": min(args.warmup, 1),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp64",
                "data": "synthetic (analytic isentropic vortex initial condition)",
                "config": {"workload": "isentropic_vortex_2d", "cells": "1024x1024", "domain": "[0,10]^2",
                           "recipe": "teno5Rusanov", "time": "SSPRK3", "cfl": 0.4, "precision": "fp64",
                           "parallelism": f"{best['cores']} processes, one row slab each"},
                "cpu_baseline": {k: best[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": round(best["value"], 4), "unit": "Mcell-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}, "wall_s": round(time.time() - t0, 1)}
        print(json.dumps(line), flush=True)
        return
    if args.all_kernels:
        print(json.dumps(run_all_kernels(args)), flush=True)
        return
    base = None
    if rank == 0 and not args.quick and not args.no_cpu_baseline:
        base = cpu_baseline(steps=3, samples=3)  # spawned before any GPU call
    from sonicsolver_b200 import replicas
    if world > 1:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    replicas.init(world, "nccl", timeout_s=120)
    out = run_ours(args, rank, world)
    if rank == 0:
        if base is not None:
            out["cpu_baseline"] = {k: base[k] for k in ("value", "unit", "cores", "kind", "sample")}
        print(json.dumps(out), flush=True)
    replicas.finish(world)


if __name__ == "__main__":
    main()
