"""Curvilinear grids on the GPU (sfg_set_metrics) against the oracle, whose
curvilinear operator is pinned bit for bit to the reference operator
(tests/test_oracle_curv.py).  Bar: 1e-12 relative L-infinity per conserved
variable per step (FP64; the device contracts to FMA)."""
import dataclasses

import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import (FLUX_OF, NG_OF, SCHEME_OF, TIME_OF, curvilinear_metrics, from_oracle, oracle_spec,
                     smooth_state, split_recipe, to_oracle)
from sonicsolver_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-12
GRIDS = {1: ((61, 1, 1), (1.0 / 60, 1.0, 1.0)), 2: ((40, 33, 1), (0.025, 0.03, 1.0)),
         3: ((14, 12, 11), (0.07, 0.08, 0.09))}


def _pair(dim, bc, recipe, time_recipe="SSPRK3", seed=0, shock=False, cfl=0.45, precision=capi.PREC_FP64):
    n, h = GRIDS[dim]
    scheme, _ = split_recipe(recipe)
    ng = NG_OF[scheme]
    bcs = (bc,) * 3
    spec = oracle_spec(dim, n, h, bcs, bcs, recipe)
    spec.metrics = curvilinear_metrics(dim, n, h, ng, seed=seed)
    s = capi.Solver(dim, n, h, bcs, bcs, recipe=recipe, time_recipe=time_recipe, cfl=cfl, precision=precision)
    s.set_metrics(np.ascontiguousarray(spec.interior(spec.metrics)))
    q = smooth_state(dim, n, seed=seed, shock=shock)
    s.upload(np.ascontiguousarray(q))
    return s, spec, q


def _solved(spec, bc):
    return (slice(None),) * 3 if bc == capi.BC_PERIODIC else tuple(
        slice(1, -1) if spec.n[d] > 1 else slice(None) for d in (2, 1, 0))


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno7Rusanov", "weno3Rusanov", "weno5Steger",
                                    "weno5LaxFriedrichs", "weno5Roe"])
def test_curvilinear_residual_matches_oracle(dim, bc, recipe):
    s, spec, q = _pair(dim, bc, recipe, seed=dim, shock=dim < 3)
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    sl = _solved(spec, bc)
    assert rel_linf(R_gpu[sl], R_ref[sl]).max() <= TOL


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("time_recipe", ["forwardEuler", "SSPRK3", "classicalRK4"])
def test_curvilinear_steps_match_oracle(dim, time_recipe):
    s, spec, q = _pair(dim, capi.BC_TRANSMISSIVE, "weno5Roe", time_recipe, seed=dim + 5)
    Q = to_oracle(spec, q)
    st = po.Stepper(spec, po.WENO5, po.ROE, TIME_OF[time_recipe])
    for _ in range(4):
        dt = po.dt(spec, Q, 0.45)
        assert abs(s.compute_dt() / dt - 1.0) <= 1e-13
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(spec.interior(Q).shape)
    assert rel_linf(got, from_oracle(spec, Q)).max() <= TOL


@pytest.mark.parametrize("dim", [1, 2])
def test_curvilinear_advance_in_graphs_matches_oracle(dim):
    s, spec, q = _pair(dim, capi.BC_PERIODIC, "weno5Rusanov", seed=11)
    Q = to_oracle(spec, q)
    dts, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, 0.05, 0.45, write_interval=0.02)
    st, dt_gpu = s.advance(0.05, write_interval=0.02, graph_steps=8, dt_capacity=4096)
    assert st.steps == len(dts)
    np.testing.assert_allclose(dt_gpu, dts, rtol=1e-12, atol=0)
    got = s.download().reshape(spec.interior(Q).shape)
    assert rel_linf(got, from_oracle(spec, Q)).max() <= 1e-11
    # conserved totals weight every node by its volume J = 1 / Jac
    J = 1.0 / spec.interior(spec.metrics)[..., 0]
    want = (from_oracle(spec, Q) * J[..., None]).reshape(-1, 5).sum(axis=0)
    np.testing.assert_allclose(s.totals(), want, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("dim", [1, 2, 3])
def test_cartesian_metrics_equal_the_uniform_kernels(dim):
    n, h = GRIDS[dim]
    bcs = (capi.BC_TRANSMISSIVE,) * 3
    q = smooth_state(dim, n, seed=4)
    a = capi.Solver(dim, n, h, bcs, bcs, recipe="weno5Rusanov")
    b = capi.Solver(dim, n, h, bcs, bcs, recipe="weno5Rusanov")
    jac = 1.0 / (h[0] * h[1] * h[2])
    M = np.zeros((n[2], n[1], n[0], 10))
    M[..., 0] = jac
    M[..., 1] = (h[1] * h[2]) * jac
    M[..., 5] = (h[0] * h[2]) * jac
    M[..., 9] = (h[0] * h[1]) * jac
    b.set_metrics(M)
    for s in (a, b):
        s.upload(np.ascontiguousarray(q))
        for _ in range(3):
            s.step(0.0)
    assert rel_linf(b.download(), a.download()).max() <= 1e-13


def test_curvilinear_with_law_ends_matches_oracle():
    """A curved 2-D channel: fixedValue inflow, zeroGradient outflow, slip and
    no-slip walls."""
    n, h = GRIDS[2]
    LAW = capi.BC_LAW
    spec = oracle_spec(2, n, h, (LAW, LAW, 0), (LAW, LAW, 0), "weno5Rusanov")
    spec.metrics = curvilinear_metrics(2, n, h, 3, seed=8)
    FV, ZG, SYM = po.LAW_FIXED_VALUE, po.LAW_ZERO_GRADIENT, po.LAW_SYMMETRY
    spec.laws = {(0, 0): po.LawSpec(FV, FV, FV, rho_value=1.1, U_value=(0.1, 0.0, 0.0), p_value=0.95),
                 (0, 1): po.LawSpec(ZG, ZG, ZG), (1, 0): po.LawSpec(ZG, SYM, ZG),
                 (1, 1): po.LawSpec(ZG, FV, ZG)}
    s = capi.Solver(2, n, h, (LAW, LAW, 0), (LAW, LAW, 0), recipe="weno5Rusanov", cfl=0.45)
    for (a, e), L in spec.laws.items():
        s.set_boundary_law(a, e, rho=L.rho, velocity=L.U, pressure=L.p, rho_value=L.rho_value,
                           velocity_value=L.U_value, pressure_value=L.p_value)
    s.set_metrics(np.ascontiguousarray(spec.interior(spec.metrics)))
    q = smooth_state(2, n, seed=8)
    s.upload(np.ascontiguousarray(q))
    # the device uploads the law ends' ghosts as copies of the boundary nodes
    frozen = dataclasses.replace(spec, bc_lo=(po.BC_FROZEN,) * 2 + (0,), bc_hi=(po.BC_FROZEN,) * 2 + (0,), laws={})
    Q = spec.empty()
    spec.interior(Q)[...] = q
    po.fill_ghosts(frozen, Q)
    Q[:, :, :3] = Q[:, :, 3:4]
    Q[:, :, -3:] = Q[:, :, -4:-3]
    Q[:, :3] = Q[:, 3:4]
    Q[:, -3:] = Q[:, -4:-3]
    st = po.Stepper(spec, po.WENO5, po.RUSANOV, po.SSPRK3)
    for _ in range(4):
        dt = po.dt(spec, Q, 0.45)
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(spec.interior(Q).shape)
    keep = np.ones(got.shape[:3], dtype=bool)
    keep[:, 0, 0] = keep[:, 0, -1] = keep[:, -1, 0] = keep[:, -1, -1] = False
    assert rel_linf(got[keep], from_oracle(spec, Q)[keep]).max() <= TOL


def test_field_layout_metrics_reach_a_frozen_ghost_face():
    """A frozen end's boundary node is advanced through the face to its ghost:
    the Field layout hands over the ghost metrics."""
    n, h = GRIDS[1]
    FR, TR = capi.BC_FROZEN, capi.BC_TRANSMISSIVE
    spec = oracle_spec(1, n, h, (FR, TR, TR), (TR, TR, TR), "weno5Rusanov")
    spec.metrics = curvilinear_metrics(1, n, h, 3, seed=3)
    s = capi.Solver(1, n, h, (FR, TR, TR), (TR, TR, TR), recipe="weno5Rusanov", cfl=0.45)
    s.set_metrics(curvilinear_metrics(1, n, h, 3, seed=3, field_layout=True), layout=capi.LAYOUT_FIELD)
    q = smooth_state(1, n, seed=3)
    s.upload(np.ascontiguousarray(q))
    Q = spec.empty()
    spec.interior(Q)[...] = q
    po.fill_ghosts(spec, Q)
    Q[0, 0, :3] = Q[0, 0, 3]
    st = po.Stepper(spec, po.WENO5, po.RUSANOV, po.SSPRK3)
    for _ in range(4):
        dt = po.dt(spec, Q, 0.45)
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(spec.interior(Q).shape)
    assert rel_linf(got[..., :-1, :], from_oracle(spec, Q)[..., :-1, :]).max() <= TOL


def test_metric_arguments_are_checked():
    n, h = GRIDS[1]
    bcs = (capi.BC_TRANSMISSIVE,) * 3
    M = curvilinear_metrics(1, n, h, 3)[:, :, 3:-3].copy()
    with pytest.raises(capi.SolverError):
        capi.Solver(1, n, h, bcs, bcs, recipe="weno5LaxWendroff").set_metrics(M)
    bad = M.copy()
    bad[0, 0, 5, 3] = np.nan
    with pytest.raises(capi.SolverError):
        capi.Solver(1, n, h, bcs, bcs).set_metrics(bad)
    zero = M.copy()
    zero[0, 0, 7:9, 1:] = 0.0       # the face (7 | 8) has no area
    with pytest.raises(capi.SolverError):
        capi.Solver(1, n, h, bcs, bcs).set_metrics(zero)


# FP32-flux / FP64-state on curvilinear grids: FP32 deviations from an FP64
# reference (each face's left node in 1-D / 3-D; the tile's first node in
# the fused 2-D tile kernel), FP32 reconstruction and flux deviation, the
# reference's flux in FP64.  Steps: the uniform FP32 path's bar, 2e-6
# relative; TENO5's cut-off decisions flip near its threshold in FP32 (max
# 1e-4, mean 1e-7).  Residuals alone are the more sensitive measure -- their
# FP32 error scales with the state's variation across a 22-node tile -- and
# are held to 5e-6.

@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "weno5Roe", "weno3Rusanov", "weno7Rusanov"])
def test_curvilinear_fp32_residual_near_oracle(dim, bc, recipe):
    s, spec, q = _pair(dim, bc, recipe, seed=dim + 20, precision=capi.PREC_FP32_FLUX)
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    sl = _solved(spec, bc)
    assert rel_linf(R_gpu[sl], R_ref[sl]).max() <= 5e-6


@pytest.mark.parametrize("dim", [1, 2, 3])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "weno5Roe", "teno5Rusanov"])
def test_curvilinear_fp32_steps_near_oracle(dim, recipe):
    s, spec, q = _pair(dim, capi.BC_PERIODIC, recipe, seed=dim + 30, precision=capi.PREC_FP32_FLUX)
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    st = po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3)
    for _ in range(4):
        dt = po.dt(spec, Q, 0.45)
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(spec.interior(Q).shape)
    err = rel_linf(got, from_oracle(spec, Q))
    if scheme == "teno5":
        assert err.max() <= 1e-4
        scale = np.abs(from_oracle(spec, Q)).reshape(-1, 5).max(axis=0)
        scale = np.where(scale > 0, scale, scale.max())
        assert (np.abs(got - from_oracle(spec, Q)).reshape(-1, 5) / scale).mean() <= 1e-7
    else:
        assert err.max() <= 2e-6


@pytest.mark.parametrize("variant", [0, 1])
@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_curvilinear_2d_face_launches_and_fused_tiles(variant, precision, bc):
    """2-D curvilinear stages: variant 0 runs the per-axis face launches,
    variant 1 the fused tile kernel; both against the oracle, through a
    residual and three steps."""
    s, spec, q = _pair(2, bc, "weno5Roe", seed=41, precision=precision)
    s.variant = variant
    Q = to_oracle(spec, q)
    R_ref = from_oracle(spec, po.rhs(spec, po.WENO5, po.ROE, Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    sl = _solved(spec, bc)
    fp64 = precision == capi.PREC_FP64
    assert rel_linf(R_gpu[sl], R_ref[sl]).max() <= (TOL if fp64 else 5e-6)
    st = po.Stepper(spec, po.WENO5, po.ROE, po.SSPRK3)
    for _ in range(3):
        dt = po.dt(spec, Q, 0.45)
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(spec.interior(Q).shape)
    assert rel_linf(got, from_oracle(spec, Q)).max() <= (TOL if fp64 else 2e-6)
