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



# ---- frozen and law ends in batches and the server

INFLOW = dict(rho=capi.LAW_FIXED_VALUE, velocity=capi.LAW_FIXED_VALUE, pressure=capi.LAW_FIXED_VALUE, rho_value=1.0,
              velocity_value=(0.3, 0.0, 0.0), pressure_value=1.0)
WALL = dict(rho=capi.LAW_ZERO_GRADIENT, velocity=capi.LAW_FIXED_VALUE, pressure=capi.LAW_ZERO_GRADIENT)
SLIP = dict(rho=capi.LAW_ZERO_GRADIENT, velocity=capi.LAW_SYMMETRY, pressure=capi.LAW_SYMMETRY)


def boundary_mix(t_end=0.04):
    """Grids with every end kind a case directory gives: a Sod tube without
    a Left condition (frozen), a tube with a fixedValue inflow and a noSlip
    wall, a 2-D box with noSlip and slip walls, and one with a
    frozen low y end, beside plain transmissive and periodic grids.
    Returns [(case, laws)]."""
    sod = cases.sod_1d(cells=600, t_end=t_end)
    sod.bc_lo = (capi.BC_FROZEN, 0, 0)
    tube = cases.sod_1d(cells=450, t_end=t_end)
    tube.bc_lo = tube.bc_hi = (capi.BC_LAW, 0, 0)
    box = cases.shock_tube_batch(count=8, seed=5, t_end=t_end, max_1d=800, max_2d=70)[-1]
    assert box.dim == 2
    walls = cases.Case(box.name + "_walls", 2, box.n, box.h, (capi.BC_LAW, capi.BC_LAW, 0),
                       (capi.BC_LAW, capi.BC_LAW, 0), box.q.copy(), box.gamma, t_end, box.cfl)
    frozen_y = cases.Case(box.name + "_frozen", 2, box.n, box.h, (0, capi.BC_FROZEN, 0), (0, 0, 0), box.q.copy(),
                          box.gamma, t_end, box.cfl)
    plain = cases.shock_tube_batch(count=3, seed=9, t_end=t_end, max_1d=700, max_2d=72)
    vortex = cases.isentropic_vortex(40, recipe="weno5Rusanov", cfl=0.5, t_end=0.1)
    return ([(sod, None), (tube, {(0, 0): INFLOW, (0, 1): WALL}),
             (walls, {(0, 0): WALL, (0, 1): SLIP, (1, 0): SLIP, (1, 1): WALL}), (frozen_y, None)] +
            [(c, None) for c in plain] + [(vortex, None)])


def solo_laws(case, laws, precision, variant):
    """The grid alone on the tile kernel of the batch's tile shape, with its
    laws."""
    s = capi.Solver(case.dim, case.n, case.h, case.bc_lo, case.bc_hi, recipe="weno5Rusanov", time_recipe="SSPRK3",
                    precision=precision, cfl=case.cfl)
    s.variant = variant if case.dim == 2 else 1
    for (axis, end), kw in (laws or {}).items():
        s.set_boundary_law(axis, end, **kw)
    s.upload(np.ascontiguousarray(case.q))
    st, _ = s.advance(case.t_end)
    out = s.download().reshape(case.q.shape), st.steps
    s.close()
    return out


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("variant", [1, 2])
def test_batch_with_frozen_and_law_ends_equals_solo(precision, variant):
    """Law and frozen ends run in the batch exactly as on a single grid: the
    same steps and the same bits (the batch runs the single-grid tile body
    and law arithmetic on the same device layout)."""
    grids = boundary_mix()
    b = capi.Batch(1 << 30, 32, recipe="weno5Rusanov", precision=precision, cfl=0.5)
    b.variant = variant
    slots = [b.add(c, laws=laws) for c, laws in grids]
    b.step(100000, graph_steps=8)
    for (c, laws), slot in zip(grids, slots):
        st = b.status(slot)
        assert not st["running"] and st["flags"] == 0, c.name
        want, steps = solo_laws(c, laws, precision, variant)
        assert st["steps"] == steps, c.name
        got = b.download(slot).reshape(c.q.shape)
        assert np.array_equal(got, want), (c.name, rel_linf(got, want))
    b.close()


def test_server_with_law_requests_equals_solo():
    grids = boundary_mix(t_end=0.03)
    srv = capi.Server(1 << 30, 8, recipe="weno5Rusanov", precision=capi.PREC_FP64, cfl=0.5, graph_steps=4)
    ids = [srv.submit(c, laws=laws) for c, laws in grids]
    srv.drain(300)
    for (c, laws), rid in zip(grids, ids):
        info = srv.poll(rid)
        assert info.state == capi.REQ_DONE, c.name
        want, steps = solo_laws(c, laws, capi.PREC_FP64, 1)
        assert info.steps == steps and np.array_equal(srv.fetch(rid).reshape(c.q.shape), want), c.name
    srv.close()


def test_law_ends_need_valid_laws():
    tube = cases.sod_1d(cells=100, t_end=0.01)
    tube.bc_lo = tube.bc_hi = (capi.BC_LAW, 0, 0)
    b = capi.Batch(1 << 28, 4, recipe="weno5Rusanov", cfl=0.5)
    with pytest.raises(capi.SolverError, match="needs its laws"):
        b.add(tube)
    bad = dict(INFLOW, rho_value=-1.0)
    with pytest.raises(capi.SolverError, match="density must be > 0"):
        b.add(tube, laws={(0, 0): bad, (0, 1): WALL})
    srv = capi.Server(1 << 28, 4, recipe="weno5Rusanov", cfl=0.5)
    with pytest.raises(capi.SolverError, match="needs its laws"):
        srv.submit(tube)
    srv.close()
    b.close()
