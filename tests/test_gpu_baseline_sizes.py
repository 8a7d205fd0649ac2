"""Parity with the CPU oracle at the benchmark workloads' full sizes.

The other parity tests run on grids of at most 64 x 48 nodes; these run the
workloads the benchmark quotes, at their sizes, against the oracle's own time
loop on the same inputs:

  * the 2-D periodic isentropic vortex, 1024^2 cells (TENO5 + Rusanov,
    SSPRK3, CFL 0.4): one step, every 2-D kernel variant, FP64 and FP32 flux;
  * the 3-D Taylor-Green vortex (WENO5 + Rusanov, SSPRK3, CFL 0.5): one step
    at 128^3, and the 256^3 residual on z-slabs (the oracle gets each slab
    with its periodic halo);
  * the seeded batch of 512 shock tubes: the largest 1-D tube, the largest
    2-D tube and a diagonal-diaphragm 2-D tube, 20 steps inside a batch;
  * a 1024^2 vortex request served beside other requests: 5 steps.

Tolerances, per conserved variable, relative L-infinity (max |a - b| over
max |b|; the three momentum components share one scale, the largest of the
three, because the Taylor-Green vortex starts with rho w = 0 exactly and one
step leaves it at ~1e-4 of the momentum scale, built from pressure
differences of a p0 = 71 background): FP64 1e-12 per step (the project's
parity bar); several steps compound it, so k steps are held to k x 1e-12,
and the time reached to 1e-12 relative.  FP32 flux: 2e-6 per step of the
FP64 oracle (the FP32-flux bar), k steps to k x 2e-6, and the time reached
to the same k x 2e-6 (after the first step the CFL step is taken on an
FP32-flux state).  The 256^3 residual is
held to the same per-step bars as the state change of one forward-Euler
stage at the CFL step, dt R, against the state's scale: the Taylor-Green
residual is a small difference of large per-axis flux differences (div u = 0
cancels the leading energy-flux terms between the axes, over a p0 = 71
background, and div(rho u) is 0 analytically), so its own maximum is no
scale for round-off.

The oracle runs for several seconds per step at these sizes, so all oracle
jobs start together in a spawned process pool when the module's first test
asks for them, and each test waits for its own.
"""
import multiprocessing as mp
import os
from concurrent.futures import ProcessPoolExecutor

import numpy as np
import pytest

import baseline_jobs as jobs
from conftest import rel_linf_vec as rel_linf
from conftest import state_scale
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-6
TGV_SLABS = ((0, 2), (127, 2), (253, 3))   # (first plane, planes): wrap below 0, middle, wrap past 255


@pytest.fixture(scope="module")
def oracle_runs():
    picks = jobs.tube_picks()
    ctx = mp.get_context("spawn")
    ex = ProcessPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1)), mp_context=ctx)
    futs = {
        "vortex": ex.submit(jobs.vortex_1024_steps, 5),
        "tgv128": ex.submit(jobs.taylor_green_steps, 128, 1),
        **{f"tube{k}": ex.submit(jobs.tube_steps, k, 20) for k in picks},
        **{f"slab{z0}": ex.submit(jobs.taylor_green_slab_residual, 256, z0, m) for z0, m in TGV_SLABS},
    }
    yield {"picks": picks, "futures": futs}
    ex.shutdown(wait=False, cancel_futures=True)


def _result(runs, key):
    return runs["futures"][key].result(timeout=900)


# ----------------------------------------------------------------- c2: vortex 1024^2

@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("variant", [0, 1, 2])
def test_vortex_1024_one_step(oracle_runs, variant, precision):
    c = cases.isentropic_vortex(1024)
    s = c.solver(precision=precision)
    s.variant = variant
    st, dts = s.advance(c.t_end, max_steps=1, dt_capacity=1)
    got = s.download().reshape(c.q.shape)
    s.close()
    ref_dts, states = _result(oracle_runs, "vortex")
    assert st.steps == 1
    assert abs(dts[0] - ref_dts[0]) <= 1e-14 * ref_dts[0]          # dt stays FP64 in both modes
    err = rel_linf(got, states[1].reshape(c.q.shape))
    assert err.max() <= (TOL64 if precision == capi.PREC_FP64 else TOL32), (variant, err)


# ----------------------------------------------------------------- c3: Taylor-Green

@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("variant", [0, 1])
def test_taylor_green_128_one_step(oracle_runs, variant, precision):
    c = cases.taylor_green(128)
    s = c.solver(precision=precision)
    s.variant = variant
    st, dts = s.advance(c.t_end, max_steps=1, dt_capacity=1)
    got = s.download().reshape(c.q.shape)
    s.close()
    ref_dts, states = _result(oracle_runs, "tgv128")
    assert abs(dts[0] - ref_dts[0]) <= 1e-14 * ref_dts[0]
    err = rel_linf(got, states[1].reshape(c.q.shape))
    assert err.max() <= (TOL64 if precision == capi.PREC_FP64 else TOL32), (variant, err)


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
def test_taylor_green_256_residual_on_slabs(oracle_runs, precision):
    N = 256
    c = cases.taylor_green(N)
    s = c.solver(precision=precision)
    R = s.residual().reshape(c.q.shape)
    dt = s.compute_dt()
    s.close()
    scale = state_scale(c.q)
    del c
    for z0, m in TGV_SLABS:
        want = _result(oracle_runs, f"slab{z0}")
        got = R[np.arange(z0, z0 + m) % N]
        err = dt * np.abs(got - want).reshape(-1, 5).max(axis=0) / scale
        assert err.max() <= (TOL64 if precision == capi.PREC_FP64 else TOL32), (z0, err)


# ----------------------------------------------------------------- c4: batched tubes

@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("variant", [1, 2])
def test_batched_tubes_20_steps(oracle_runs, variant, precision):
    steps = 20
    tubes = cases.shock_tube_batch(count=jobs.TUBE_COUNT, seed=jobs.TUBE_SEED, t_end=0.15)
    picks = oracle_runs["picks"]
    b = capi.Batch(4 << 30, 16, recipe="weno5Rusanov", precision=precision, cfl=0.5)
    b.variant = variant
    # the three checked tubes among other tubes of the same batch
    others = [k for k in range(0, jobs.TUBE_COUNT, 37) if k not in picks][:6]
    slots = {k: b.add(tubes[k], max_steps=steps) for k in list(picks) + others}
    b.step(steps + 5, graph_steps=8)
    tol = steps * (TOL64 if precision == capi.PREC_FP64 else TOL32)
    for k in picks:
        c = tubes[k]
        st = b.status(slots[k])
        ref_dts, states = _result(oracle_runs, f"tube{k}")
        assert st["steps"] == steps and not st["running"] and st["flags"] == 0
        t_tol = 1e-12 if precision == capi.PREC_FP64 else tol
        assert abs(st["time"] - ref_dts.sum()) <= t_tol * ref_dts.sum(), k
        err = rel_linf(b.download(slots[k]).reshape(c.q.shape), states[steps].reshape(c.q.shape))
        assert err.max() <= tol, (k, c.name, err)
    b.close()


# ----------------------------------------------------------------- c5: a served 1024^2 request

@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
def test_served_vortex_1024_five_steps(oracle_runs, precision):
    steps = 5
    big = cases.isentropic_vortex(1024)
    small = [cases.isentropic_vortex(n) for n in (64, 96, 128)]
    srv = capi.Server(8 << 30, 8, recipe="teno5Rusanov", precision=precision, cfl=0.4, graph_steps=2)
    ids = [srv.submit(c, max_steps=40) for c in small[:2]]
    rid = srv.submit(big, max_steps=steps)                   # arrives while the others run
    ids.append(srv.submit(small[2], max_steps=40))
    srv.drain(600)
    info = srv.poll(rid)
    assert info.state == capi.REQ_DONE and info.steps == steps
    got = srv.fetch(rid).reshape(big.q.shape)
    for i in ids:
        assert srv.poll(i).state == capi.REQ_DONE
    srv.close()
    ref_dts, states = _result(oracle_runs, "vortex")
    tol = steps * (TOL64 if precision == capi.PREC_FP64 else TOL32)
    assert abs(info.time - ref_dts.sum()) <= (1e-12 if precision == capi.PREC_FP64 else tol) * ref_dts.sum()
    err = rel_linf(got, states[steps].reshape(big.q.shape))
    assert err.max() <= tol, err
