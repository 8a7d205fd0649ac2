"""The N > 1 path (replicas, one process per GPU) on CPU: two gloo ranks take
the same collective steps bench.py takes -- a barrier on each side of the
timed region, the maximum of the ranks' times -- and the whole-job rate is
the work of both ranks over the slower rank's time.  Rank 0 then keeps
working on its own (the one-GPU legs) while rank 1 leaves: nothing waits."""
import os
import socket
import time

import pytest
import torch.multiprocessing as mp

from sonicsolver_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    r, w, lr = replicas.world_info()
    assert (r, w, lr) == (rank, world, rank)
    replicas.init(w, "gloo", timeout_s=30)
    replicas.barrier(w)
    ms = 10.0 + 5.0 * rank                     # this rank's device time
    replicas.barrier(w)
    ms_max = replicas.max_over_ranks(ms, w)
    rate = replicas.whole_job_rate(1000.0, ms_max, w)
    if rank == 0:
        time.sleep(0.5)                        # rank 0's own legs after the collectives
    replicas.finish(w)
    out.put((rank, ms_max, rate))


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(90)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(2))
    for rank, ms_max, rate in res:
        assert ms_max == 15.0                  # the slower rank's 15 ms
        assert rate == pytest.approx(2 * 1000.0 / 15e-3)


def test_single_rank_needs_no_process_group():
    assert replicas.max_over_ranks(3.5, 1) == 3.5
    replicas.barrier(1)
    replicas.init(1)
    replicas.finish(1)
    assert replicas.whole_job_rate(500.0, 10.0, 1) == pytest.approx(5e4)
