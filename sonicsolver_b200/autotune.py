"""Tile-shape autotuner.

Picks the stage-operator kernel variant by timing the candidates on the
device, per (GPU model, dimension, size class, recipe, precision):

  * single grids: variant 0 (one sweep launch per axis), 1 (32 x 15 tiles,
    511-node 1-D tiles, or 3-D 16 x 15 columns marching in z), 2 (22 x 22
    tiles, 2-D only), each timed with
    sfg_time_sweeps (CUDA events on the solver's stream, stage 0 repeated);
    a 1-D tile win selects 1-D variant 2, which runs the same tiles for
    single stages and adds the whole-run cluster kernel to sfg_advance;
  * batches: 2-D work-item tile 32 x 15 or 22 x 22, timed over a few batch
    steps of a sample of the batch's grids.

Results are cached in a JSON table (default ``~/.cache/sonicsolver_b200/
tuning.json``, or $SFG_TUNING_FILE) so the search runs once per shape class.
Every variant computes the same result (FP64: identical to round-off; FP32:
the per-tile reference changes the rounding), so tuning never changes the
numerics beyond that.
"""
from __future__ import annotations

import json
import math
import os
import threading

from . import capi

_LOCK = threading.Lock()


def _table_path() -> str:
    p = os.environ.get("SFG_TUNING_FILE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "sonicsolver_b200", "tuning.json")


def _load() -> dict:
    try:
        with open(_table_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table: dict) -> None:
    path = _table_path()
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass  # a read-only home only loses the cache


def _gpu_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:
        return "unknown-gpu"


def size_class(nodes: int) -> int:
    """Power-of-four bucket of the node count."""
    return int(round(math.log(max(nodes, 1), 4)))


def candidates(dim: int):
    return {1: [0, 1], 2: [0, 1, 2], 3: [0, 1]}[dim]


def tune_solver(solver: "capi.Solver", recipe: str, precision: int, repeats: int = 5, use_cache: bool = True) -> dict:
    """Times the variants on `solver`'s current state and selects the fastest
    (the solver keeps it).  Returns {variant: ms per stage, 'best': v}."""
    nodes = int(solver.n[0] * solver.n[1] * solver.n[2])
    key = f"{_gpu_name()}|solver|{solver.dim}|{size_class(nodes)}|{recipe}|{precision}"
    with _LOCK:
        table = _load() if use_cache else {}
        if key in table:
            solver.variant = table[key]["best"]
            return table[key]
    dt = solver.compute_dt()
    result = {}
    for v in candidates(solver.dim):
        solver.variant = v
        solver.time_sweeps(dt, stage=0, repeats=1)          # warm-up (lazy module load)
        result[str(v)] = sum(solver.time_sweeps(dt, stage=0, repeats=repeats))
    best = int(min(result, key=result.get))
    if solver.dim == 1 and best == 1:
        best = 2  # the same stage operator, plus the whole-run cluster kernel
    solver.variant = best
    entry = {"ms_per_stage": result, "best": best}
    with _LOCK:
        table = _load()
        table[key] = entry
        _store(table)
    return entry


def tune_batch(make_batch, sample_cases, recipe: str, precision: int, steps: int = 6, use_cache: bool = True) -> int:
    """Times batch tile shapes 1 and 2 on `sample_cases` (a callable
    make_batch() -> capi.Batch builds an empty batch) and returns the faster."""
    import torch
    cells = sum(c.cells for c in sample_cases)
    key = f"{_gpu_name()}|batch|{size_class(cells)}|{recipe}|{precision}"
    with _LOCK:
        table = _load() if use_cache else {}
        if key in table:
            return table[key]["best"]
    times = {}
    for v in (1, 2):
        b = make_batch()
        b.variant = v
        for c in sample_cases:
            b.add(c)
        b.step(2, graph_steps=2)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        b.step(steps, graph_steps=steps)
        e1.record()
        torch.cuda.synchronize()
        times[str(v)] = e0.elapsed_time(e1) / steps
        b.close()
    best = int(min(times, key=times.get))
    with _LOCK:
        table = _load()
        table[key] = {"ms_per_step": times, "best": best}
        _store(table)
    return best
