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


def _rank_work(rank, world, port, out):
    """A replica rank with real solver work: it steps its own seeded tube with
    the CPU oracle (the GPU ranks step theirs with the provider), then takes
    the bench's collectives: barrier, max over ranks of the times."""
    import numpy as np
    import pyoracle as po
    from helpers import oracle_spec, to_oracle, from_oracle
    from sonicsolver_b200 import cases
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    replicas.init(world, "gloo", timeout_s=30)
    c = cases.shock_tube_batch(count=world, seed=5, t_end=0.01, max_1d=600, max_2d=72)[rank]
    spec = oracle_spec(c, recipe=c.recipe)
    Q = to_oracle(spec, c.q)
    replicas.barrier(world)
    t0 = time.perf_counter()
    dts, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, c.t_end, c.cfl)
    ms = (time.perf_counter() - t0) * 1e3
    replicas.barrier(world)
    ms_max = replicas.max_over_ranks(ms, world)
    replicas.finish(world)
    out.put((rank, ms, ms_max, len(dts), tf, np.ascontiguousarray(from_oracle(spec, Q)).tobytes()))


@pytest.mark.timeout(180)
def test_two_gloo_ranks_step_their_own_grids():
    """Each rank's result equals the same grid stepped by one process alone,
    and both ranks report the slower rank's time."""
    import numpy as np
    import pyoracle as po
    from helpers import oracle_spec, to_oracle, from_oracle
    from sonicsolver_b200 import cases
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_work, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=150) for _ in range(world))
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    slowest = max(r[1] for r in res)
    for rank, ms, ms_max, steps, tf, state in res:
        assert ms_max == pytest.approx(slowest)
        c = cases.shock_tube_batch(count=world, seed=5, t_end=0.01, max_1d=600, max_2d=72)[rank]
        spec = oracle_spec(c, recipe=c.recipe)
        Q = to_oracle(spec, c.q)
        dts, tf_alone = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, c.t_end, c.cfl)
        assert steps == len(dts) and tf == tf_alone
        alone = np.ascontiguousarray(from_oracle(spec, Q))
        assert np.array_equal(np.frombuffer(state, dtype=np.float64).reshape(alone.shape), alone)
