"""Parity of the sm_100a FP64 path with the CPU oracle, through the C ABI.

Bar: <= 1e-12 relative L-infinity per conserved variable per step (operator,
stage and step level), on seeded smooth and discontinuous states, 1-D / 2-D /
3-D, transmissive and periodic ends, every provided recipe and time recipe.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import (FLUX_OF, SCHEME_OF, TIME_OF, from_oracle, oracle_spec, smooth_state, split_recipe,
                     to_oracle)
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

TOL = 1e-12

GRIDS = [
    (1, (61, 1, 1), (0.013, 1.0, 1.0)),
    (2, (37, 29, 1), (0.021, 0.017, 1.0)),
    (3, (14, 12, 11), (0.05, 0.06, 0.07)),
]
RECIPES = ["weno5Rusanov", "teno5Rusanov", "weno5Roe", "teno5Roe", "weno3Rusanov", "weno7Rusanov"]


def _pair(dim, n, h, bc, recipe, time_recipe="SSPRK3", shock=False, seed=0):
    bcs = (bc,) * 3
    q = smooth_state(dim, n, seed=seed, shock=shock)
    spec = oracle_spec(dim, n, h, bcs, bcs, recipe)
    s = capi.Solver(dim, n, h, bcs, bcs, recipe=recipe, time_recipe=time_recipe, cfl=0.5)
    s.upload(np.ascontiguousarray(q))
    return s, spec, q


@pytest.mark.parametrize("recipe", RECIPES)
@pytest.mark.parametrize("dim,n,h", GRIDS)
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
@pytest.mark.parametrize("shock", [False, True])
def test_residual_parity(recipe, dim, n, h, bc, shock):
    s, spec, q = _pair(dim, n, h, bc, recipe, shock=shock)
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    # compare on solved nodes: transmissive boundary nodes are not advanced
    # (the GPU reports 0 there; the oracle evaluates them anyway)
    sl = tuple(slice(1, -1) if (d < dim and bc == capi.BC_TRANSMISSIVE) else slice(None) for d in (2, 1, 0))
    err = rel_linf(R_gpu[sl], R_ref[sl])
    assert err.max() <= TOL, (recipe, dim, bc, shock, err)


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno7Rusanov", "weno3Rusanov"])
@pytest.mark.parametrize("n", [(37, 29, 1), (64, 48, 1), (9, 40, 1)])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_2d_kernel_variants_match_oracle(variant, recipe, n, bc):
    """Axis sweeps (0) and fused tile kernels (1: 32x15, 2: 22x22) on grids
    smaller than, equal to and not a multiple of a tile, including periodic
    axes shorter than the tile halo reach."""
    h = (0.03, 0.02, 1.0)
    s, spec, q = _pair(2, n, h, bc, recipe, shock=True, seed=9)
    s.variant = variant
    assert s.variant == variant
    scheme, flux = split_recipe(recipe)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], to_oracle(spec, q)))
    R_gpu = s.residual().reshape(R_ref.shape)
    sl = tuple(slice(1, -1) if (d < 2 and bc == capi.BC_TRANSMISSIVE) else slice(None) for d in (2, 1, 0))
    assert rel_linf(R_gpu[sl], R_ref[sl]).max() <= TOL
    # one SSPRK3 step through the same variant
    Q = to_oracle(spec, q)
    dt = po.dt(spec, Q, 0.5)
    po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3).step(Q, dt)
    s.step(dt)
    assert rel_linf(s.download().reshape(q.shape), from_oracle(spec, Q)).max() <= TOL


def test_variants_by_dimension():
    s, _, _ = _pair(1, (61, 1, 1), (0.013, 1.0, 1.0), capi.BC_PERIODIC, "weno5Rusanov")
    assert s.variant == 2            # 1-D tiles + the whole-run cluster kernel
    s.variant = 1
    with pytest.raises(capi.SolverError):
        s.variant = 3
    s3, _, _ = _pair(3, (14, 12, 11), (0.05, 0.06, 0.07), capi.BC_PERIODIC, "weno5Rusanov")
    assert s3.variant == 0
    s3.variant = 1                  # 3-D z-marching tiles
    assert s3.variant == 1
    with pytest.raises(capi.SolverError):
        s3.variant = 2


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno7Rusanov", "weno3Rusanov"])
@pytest.mark.parametrize("n", [61, 511, 512, 1300])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_1d_kernel_variants_match_oracle(variant, recipe, n, bc):
    """1-D sweeps (0) and 511-node tiles (1), grids below, at and above a tile."""
    s, spec, q = _pair(1, (n, 1, 1), (1.0 / n, 1.0, 1.0), bc, recipe, shock=True, seed=4)
    s.variant = variant
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    sl = (slice(None), slice(None), slice(1, -1) if bc == capi.BC_TRANSMISSIVE else slice(None))
    assert rel_linf(R_gpu[sl], R_ref[sl]).max() <= TOL
    dt = po.dt(spec, Q, 0.5)
    po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3).step(Q, dt)
    s.step(dt)
    assert rel_linf(s.download().reshape(q.shape), from_oracle(spec, Q)).max() <= TOL


@pytest.mark.parametrize("time_recipe", ["forwardEuler", "SSPRK3", "classicalRK4"])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Rusanov", "weno5Roe"])
@pytest.mark.parametrize("dim,n,h", GRIDS)
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_stage_and_step_parity(time_recipe, recipe, dim, n, h, bc):
    s, spec, q = _pair(dim, n, h, bc, recipe, time_recipe, shock=True, seed=3)
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    dt_ref = po.dt(spec, Q, 0.5)
    dt_gpu = s.compute_dt()
    assert abs(dt_gpu - dt_ref) <= 1e-14 * dt_ref
    st = po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], TIME_OF[time_recipe])
    stages = {"forwardEuler": 1, "SSPRK3": 3, "classicalRK4": 4}[time_recipe]
    for step in range(3):
        for k in range(stages):
            st.stage(Q, dt_ref, k)
            s.stage(k, dt_ref)
            if k < stages - 1:
                continue
        got = s.download().reshape(from_oracle(spec, Q).shape)
        err = rel_linf(got, from_oracle(spec, Q))
        assert err.max() <= TOL, (time_recipe, recipe, dim, bc, step, err)
        # continue from the GPU state so each step is compared on equal input
        Q = to_oracle(spec, got)


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Rusanov"])
def test_stage_arithmetic_with_given_residual(recipe):
    """Stage combination alone (SF_explicit.cpp:193-238): exact agreement."""
    dim, n, h = GRIDS[1]
    for tr in ("forwardEuler", "SSPRK3", "classicalRK4"):
        s, spec, q = _pair(dim, n, h, capi.BC_PERIODIC, recipe, tr)
        rng = np.random.default_rng(7)
        stages = {"forwardEuler": 1, "SSPRK3": 3, "classicalRK4": 4}[tr]
        Rs = [rng.standard_normal(q.shape) * 0.1 for _ in range(stages)]
        dt = 0.01
        q0 = q.copy()
        cur = q.copy()
        K = None
        for k in range(stages):
            s.stage_with_residual(k, dt, Rs[k])
            r = Rs[k]
            if tr == "forwardEuler":
                cur = cur - dt * r
            elif tr == "SSPRK3":
                base, inc = [(0.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0)][k]
                cur = base * q0 + inc * (cur - dt * r)
            else:
                if k == 0:
                    K = r.copy()
                elif k < 3:
                    K = K + 2.0 * r
                cur = q0 - [0.5, 0.5, 1.0][k] * dt * r if k < 3 else q0 - dt / 6.0 * (K + 1.0 * r)
        got = s.download().reshape(q.shape)
        assert rel_linf(got, cur).max() <= 1e-15, tr


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Rusanov"])
def test_advance_matches_oracle_time_loop(recipe):
    """sfg_advance (device dt + graph) vs the oracle's Time::Driver loop on a
    short Sod run: same dt sequence and state."""
    c = cases.sod_1d(200, recipe=recipe, t_end=0.05)
    spec = oracle_spec(c, recipe=recipe)
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, c.q)
    dts_ref, tf = po.advance(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3, Q, 0.05, 0.5, write_interval=0.02)
    s = c.solver()
    st, dts = s.advance(0.05, write_interval=0.02, graph_steps=8, dt_capacity=10000)
    assert st.steps == len(dts_ref)
    np.testing.assert_allclose(dts, dts_ref, rtol=1e-11, atol=0)
    assert abs(st.time - tf) <= 1e-14
    got = s.download().reshape(from_oracle(spec, Q).shape)
    assert rel_linf(got, from_oracle(spec, Q)).max() <= 1e-10


def test_field_layout_round_trip():
    dim, n, h = GRIDS[1]
    s, spec, q = _pair(dim, n, h, capi.BC_TRANSMISSIVE, "weno5Rusanov")
    f = s.download(capi.LAYOUT_FIELD)
    ng = 3
    F = f.reshape(n[2] + 2 * ng, n[1] + 2 * ng, n[0] + 2 * ng, 5)
    inner = F[ng:ng + n[2], ng:ng + n[1], ng:ng + n[0]]
    # boundary nodes carry their inner neighbour (transmissive commit fill)
    np.testing.assert_array_equal(inner[:, 1:-1, 1:-1], q[:, 1:-1, 1:-1])
    s2 = capi.Solver(dim, n, h, (0, 0, 0), (0, 0, 0))
    s2.upload(np.ascontiguousarray(f), layout=capi.LAYOUT_FIELD)
    np.testing.assert_array_equal(s2.download().reshape(q.shape)[:, 1:-1, 1:-1], q[:, 1:-1, 1:-1])


def test_invalid_state_reports_error():
    """A negative-pressure input is reported through the status word and the
    return code (the reference exits the process on it)."""
    dim, n, h = GRIDS[0]
    s, spec, q = _pair(dim, n, h, capi.BC_TRANSMISSIVE, "weno5Rusanov")
    bad = q.copy()
    bad[0, 0, 30, 4] = -1.0  # negative total energy -> p < 0
    s.upload(np.ascontiguousarray(bad))
    with pytest.raises(capi.SolverError) as e:
        s.step(1e-4)
    assert e.value.code == capi.ERR_STATE
    assert s.status() != 0
