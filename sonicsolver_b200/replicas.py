"""Replica runs across GPUs: one process per GPU under torch.distributed, each
rank advancing its own independent grids (a single grid does not shard in
this provider; batched and served instances are independent units).  There
is no data-path collective.  The only collectives are a barrier on each
side of a timed region and the maximum of the ranks' device times, and
every rank takes them in the same order.  The whole-job throughput is the
work of all ranks over the slowest rank's time.

The helpers run on any backend: NCCL on GPUs (tensors on the rank's
device), gloo on CPU (the multi-process tests)."""
from __future__ import annotations

import os
from datetime import timedelta


def world_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(world: int, backend: str = "nccl", timeout_s: float = 120.0) -> None:
    """Joins the process group when there is more than one rank.  The short
    timeout makes a rank that waits for a missing peer end with an error."""
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """The largest x over all ranks (the slowest rank's time)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, ms_max: float, world: int) -> float:
    """Units per second of the whole job: every rank's units over the
    slowest rank's milliseconds (weak scaling: per-rank work is fixed)."""
    return units_per_rank * world / (ms_max * 1e-3)
