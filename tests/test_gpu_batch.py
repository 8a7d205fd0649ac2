"""Batched and served forms: every grid's result must be the same in the mix
as alone (single-grid solver, same numerics) -- tolerance 1e-12 relative
L-infinity per variable, the parity tolerance of the other GPU tests; step
counts must match exactly."""
import re
import time

import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

TOL = 1e-12


def mix(seed=3, t_end=0.03):
    """A small seeded mix: 1-D tubes of uneven length, 2-D slanted tubes, a
    periodic vortex."""
    tubes = cases.shock_tube_batch(count=8, seed=seed, t_end=t_end, max_1d=1500, max_2d=90)
    vortex = cases.isentropic_vortex(48, recipe="weno5Rusanov", cfl=0.5, t_end=0.2)
    return tubes + [vortex]


def solo(case, precision=capi.PREC_FP64, recipe="weno5Rusanov", variant=1):
    """The same grid alone, on the tile kernel of the batch's tile shape."""
    s = capi.Solver(case.dim, case.n, case.h, case.bc_lo, case.bc_hi, recipe=recipe, time_recipe="SSPRK3",
                    precision=precision, cfl=case.cfl)
    if case.dim == 2:
        s.variant = variant
    s.upload(np.ascontiguousarray(case.q))
    st, _ = s.advance(case.t_end)
    return s.download().reshape(case.q.shape), st.steps


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("variant", [1, 2])
def test_batch_results_equal_solo(precision, variant):
    cs = mix()
    b = capi.Batch(1 << 30, 64, recipe="weno5Rusanov", precision=precision, cfl=0.5)
    b.variant = variant
    slots = [b.add(c) for c in cs]
    b.step(100000, graph_steps=8)
    for c, slot in zip(cs, slots):
        st = b.status(slot)
        assert not st["running"] and st["flags"] == 0
        assert abs(st["time"] - c.t_end) < 1e-12
        want, steps = solo(c, precision, variant=variant)
        assert st["steps"] == steps, c.name
        assert rel_linf(b.download(slot), want).max() <= TOL, c.name


def mixed_recipes(seed=13):
    """Grids that each carry their own numerics, as reference case
    directories do: tubes on WENO5 / WENO3 with Rusanov or Roe and TENO5 with
    Roe (CFL 0.5), a TENO5 + Rusanov vortex at CFL 0.4 (the vortex workload's
    numerics), a WENO7 vortex at CFL 0.45 with a maxDeltaT.  Each tube's
    recipe is one the oracle's time loop runs to t_end on that tube (WENO3
    drives some of these tubes to p < 0, as the reference does)."""
    tubes = cases.shock_tube_batch(count=8, seed=seed, t_end=0.03, max_1d=1500, max_2d=90)
    recipes = ("weno5Rusanov", "weno5Roe", "weno3Rusanov", "teno5Roe", "weno5Roe", "teno5Roe", "teno5Roe",
               "weno5Rusanov")
    for c, r in zip(tubes, recipes):
        c.recipe = r
    vortices = [cases.isentropic_vortex(48, recipe="teno5Rusanov", cfl=0.4, t_end=0.2),
                cases.isentropic_vortex(40, recipe="weno7Rusanov", cfl=0.45, t_end=0.15)]
    vortices[1].meta["max_dt"] = 2.5e-3
    return tubes + vortices


def solo_own(case, precision, variant):
    """The grid alone with its own numerics."""
    s = capi.Solver(case.dim, case.n, case.h, case.bc_lo, case.bc_hi, recipe=case.recipe, time_recipe="SSPRK3",
                    precision=precision, cfl=case.cfl, max_dt=case.meta.get("max_dt", 0.0))
    if case.dim == 2:
        s.variant = variant
    s.upload(np.ascontiguousarray(case.q))
    st, _ = s.advance(case.t_end)
    return s.download().reshape(case.q.shape), st.steps


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("variant", [1, 2])
def test_batch_with_per_grid_recipes_equals_solo(precision, variant):
    """One batch, five recipes and three CFL numbers: each grid's result and
    step count equal the same grid run alone with its own numerics."""
    cs = mixed_recipes()
    b = capi.Batch(1 << 30, 64, recipe="weno5Rusanov", precision=precision, cfl=0.5)
    b.variant = variant
    slots = [b.add(c, recipe=c.recipe, cfl=c.cfl, max_dt=c.meta.get("max_dt")) for c in cs]
    b.step(100000, graph_steps=8)
    for c, slot in zip(cs, slots):
        st = b.status(slot)
        assert not st["running"] and st["flags"] == 0, c.name
        assert abs(st["time"] - c.t_end) < 1e-12
        want, steps = solo_own(c, precision, variant)
        assert st["steps"] == steps, (c.name, c.recipe)
        assert rel_linf(b.download(slot), want).max() <= TOL, (c.name, c.recipe)


def test_server_with_per_request_recipes_equals_solo():
    """Staggered arrivals of requests with their own recipes and CFL numbers,
    fewer slots than requests: each result equals the grid alone."""
    cs = mixed_recipes()
    srv = capi.Server(1 << 30, 5, recipe="weno5Rusanov", graph_steps=4)
    ids = []
    for c in cs:
        ids.append(srv.submit(c, recipe=c.recipe, cfl=c.cfl, max_dt=c.meta.get("max_dt")))
        time.sleep(0.002)
    srv.drain(300)
    for rid, c in zip(ids, cs):
        info = srv.poll(rid)
        assert info.state == capi.REQ_DONE, (c.name, c.recipe)
        want, steps = solo_own(c, capi.PREC_FP64, 1)
        assert info.steps == steps
        assert rel_linf(srv.fetch(rid), want).max() <= TOL
    srv.close()


def test_per_grid_numerics_are_checked():
    """A grid's own numerics must keep the batch's time recipe and precision
    and name a recipe with a batched kernel; the server checks at submit."""
    import ctypes
    c = cases.sod_1d(100, t_end=0.01)
    b = capi.Batch(64 << 20, 4)
    g = capi.grid_desc(c.dim, c.n, c.h, c.bc_lo, c.bc_hi)
    q = np.ascontiguousarray(c.q)
    slot = ctypes.c_int()
    for kw in ({"time_recipe": "classicalRK4"}, {"precision": capi.PREC_FP32_FLUX}, {"recipe": "weno5Steger"},
               {"cfl": float("nan")}):
        nm = capi.numerics_desc(**{**b.defaults, **kw})
        code = capi.lib().sfg_batch_add_ex(b._h, ctypes.byref(g), ctypes.byref(nm),
                                           q.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 0.01, 0,
                                           ctypes.byref(slot))
        assert code == capi.ERR_ARG, kw
    assert b.info()["live"] == 0
    b.close()
    srv = capi.Server(64 << 20, 2)
    with pytest.raises(capi.SolverError) as e:
        srv.submit(c, recipe="teno5LaxWendroff")
    assert e.value.code == capi.ERR_ARG
    srv.close()


def test_continuous_batching_add_and_remove_between_steps():
    cs = mix(seed=5)
    b = capi.Batch(1 << 30, 16)
    first = {b.add(c): c for c in cs[:4]}
    b.step(10, graph_steps=4)
    later = {b.add(c): c for c in cs[4:]}
    done = {}
    for _ in range(10000):
        active = b.step(8, graph_steps=8)
        for slot in list(first) + list(later):
            if slot in done:
                continue
            st = b.status(slot)
            if not st["running"]:
                done[slot] = (b.download(slot), st["steps"])
                b.remove(slot)
        if active == 0 and len(done) == len(cs):
            break
    assert len(done) == len(cs)
    for slot, c in {**first, **later}.items():
        want, steps = solo(c)
        got, got_steps = done[slot]
        assert got_steps == steps
        assert rel_linf(got, want).max() <= TOL
    assert b.info()["used"] == 0 and b.info()["live"] == 0


def test_budget_rejects_and_others_continue():
    c = cases.sod_1d(400, t_end=0.02)
    b = capi.Batch(1 << 20, 64)   # 1 MiB, more slots than fit
    need = b.instance_bytes(c)
    fits = (1 << 20) // need
    slots = [b.add(c) for _ in range(fits)]
    with pytest.raises(capi.SolverError) as e:
        b.add(c)
    assert e.value.code == capi.ERR_BUDGET
    b.step(100000)
    want, steps = solo(c)
    for s in slots:
        assert rel_linf(b.download(s), want).max() <= TOL


def test_failing_grid_is_isolated():
    """A grid that goes invalid stops with its flags set; the others finish
    exactly as alone (the reference would exit the whole process)."""
    cs = mix(seed=7)
    bad = cases.sod_1d(300, t_end=0.03)
    bad.q[0, 0, 150, 4] = -1.0
    b = capi.Batch(1 << 30, 32)
    slots = [b.add(c) for c in cs]
    bad_slot = b.add(bad)
    b.step(100000)
    st = b.status(bad_slot)
    assert st["flags"] != 0 and not st["running"]
    for c, slot in zip(cs, slots):
        want, steps = solo(c)
        assert b.status(slot)["steps"] == steps
        assert rel_linf(b.download(slot), want).max() <= TOL


def test_server_results_equal_solo_with_staggered_arrivals():
    cs = mix(seed=11)
    srv = capi.Server(1 << 30, 6, graph_steps=4)   # fewer slots than requests: queueing
    ids = []
    for c in cs:
        ids.append(srv.submit(c))
        time.sleep(0.002)                             # arrivals while others run
    srv.drain(300)
    for rid, c in zip(ids, cs):
        info = srv.poll(rid)
        assert info.state == capi.REQ_DONE
        assert info.submit_s <= info.admit_s <= info.finish_s
        want, steps = solo(c)
        assert info.steps == steps
        assert rel_linf(srv.fetch(rid), want).max() <= TOL
    srv.close()


def test_server_cancel_and_oversized_request():
    c = cases.isentropic_vortex(48, t_end=5.0)
    srv = capi.Server(64 << 20, 1, graph_steps=4)
    a = srv.submit(c)
    b = srv.submit(c)          # waits: one slot
    srv.cancel(b)
    srv.cancel(a)
    srv.drain(120)
    assert srv.poll(b).state == capi.REQ_CANCELLED
    assert srv.poll(a).state == capi.REQ_CANCELLED
    big = cases.isentropic_vortex(2048, t_end=1.0)
    with pytest.raises(capi.SolverError) as e:
        srv.submit(big)       # more than the whole budget
    assert e.value.code == capi.ERR_BUDGET
    srv.close()


# A double rarefaction close to vacuum (rho ~ 3.6, u = -0.645 | +0.755,
# p = 0.103 | 0.284): the scheme drives p below zero within a few steps, and
# the reference stops on it (requirePhysicalState).  The GPU paths must stop
# in the step where the oracle's time loop stops, and count that step.
DOUBLE_RAREFACTION = dict(left=(3.569, -0.645, 0.103), right=(3.701, 0.755, 0.284))


def _oracle_failure_step(c):
    """Steps the oracle completes before the step that goes invalid."""
    spec = po.GridSpec(dim=c.dim, n=tuple(c.n), ng=3, h=tuple(c.h), bc_lo=tuple(c.bc_lo), bc_hi=tuple(c.bc_hi),
                       gamma=c.gamma)
    Q = spec.empty()
    spec.interior(Q)[...] = c.q.reshape(spec.interior(Q).shape)
    po.fill_ghosts(spec, Q)
    with pytest.raises(po.OracleError) as e:
        po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, 1e9, c.cfl, max_steps=2000)
    return int(re.search(r"after (\d+) steps", str(e.value)).group(1))


@pytest.mark.parametrize("variant", [1, 2])
def test_near_vacuum_stops_where_the_oracle_stops(variant):
    """Single grid: the graph path (1) and the whole-run cluster kernel (2)."""
    c = cases.sod_1d(200, t_end=1e9, **DOUBLE_RAREFACTION)
    done = _oracle_failure_step(c)
    s = c.solver()
    s.variant = variant
    with pytest.raises(capi.SolverError) as e:
        s.advance(1e9, max_steps=2000, graph_steps=16)
    assert e.value.code == capi.ERR_STATE
    assert s.time()[1] == done + 1


def test_near_vacuum_request_stops_in_the_mix_where_the_oracle_stops():
    """A 2-D double rarefaction (a slanted tube of the seeded generator) in a
    batch: it stops at the oracle's step, the others finish as alone."""
    tube = cases.shock_tube_batch(count=2, seed=557824790, t_end=1e9, max_2d=211)[1]
    assert tube.dim == 2
    done = _oracle_failure_step(tube)
    others = mix(seed=5)
    b = capi.Batch(1 << 30, 32)
    slots = [b.add(c) for c in others]
    bad = b.add(tube)
    b.step(100000)
    st = b.status(bad)
    assert st["flags"] != 0 and not st["running"]
    assert st["steps"] == done + 1
    for c, slot in zip(others, slots):
        want, steps = solo(c)
        assert b.status(slot)["steps"] == steps
        assert rel_linf(b.download(slot), want).max() <= TOL

