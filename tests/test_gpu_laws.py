"""Physical boundary laws on the GPU (SFG_BC_LAW ends: fixedValue /
zeroGradient / symmetry for density, velocity and pressure) against the
oracle, whose laws are pinned bit for bit to the reference's own law code
(tests/test_oracle_laws.py).

Nodes on two or more non-periodic boundary planes (box edges and corners)
are read by no stencil of a solved node; the device does not maintain them,
so the comparisons leave them out."""
import dataclasses

import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import FLUX_OF, SCHEME_OF, TIME_OF, from_oracle, oracle_spec, smooth_state, split_recipe
from sonicsolver_b200 import capi

pytestmark = pytest.mark.gpu

ZG, FV, SYM = po.LAW_ZERO_GRADIENT, po.LAW_FIXED_VALUE, po.LAW_SYMMETRY
LAW, TR, PER = capi.BC_LAW, capi.BC_TRANSMISSIVE, capi.BC_PERIODIC

INFLOW = (FV, FV, FV)          # supersonic-style inflow: rho, U, p prescribed
WALL = (ZG, FV, ZG)            # no-slip wall: U = 0
SLIP = (ZG, SYM, ZG)           # symmetry plane / slip wall
OUTFLOW = (ZG, ZG, ZG)         # zeroGradient with energy rebuilt from pressure
SUBSONIC_IN = (ZG, FV, FV)     # U and p prescribed, density extrapolated


def _law_spec(kinds, axis, end):
    return po.LawSpec(*kinds, rho_value=1.1 + 0.05 * axis, U_value=(0.0, 0.0, 0.0) if kinds == WALL else
                      (0.12 - 0.05 * end, -0.04 * axis, 0.02), p_value=0.97 + 0.02 * end)


def _setup(dim, n, bc_lo, bc_hi, kinds, recipe="weno5Rusanov", time_recipe="SSPRK3", precision=capi.PREC_FP64,
           seed=0, shock=False, variant=None):
    """GPU solver and oracle spec with the same laws; `kinds[(axis, end)]`
    gives the (rho, U, p) laws of each law end."""
    h = tuple(1.0 / n[d] if d < dim else 1.0 for d in range(3))
    spec = oracle_spec(dim, n, h, bc_lo, bc_hi, recipe)
    spec.laws = {ae: _law_spec(k, *ae) for ae, k in kinds.items()}
    s = capi.Solver(dim, n, h, bc_lo, bc_hi, recipe=recipe, time_recipe=time_recipe, precision=precision, cfl=0.45)
    for (axis, end), L in spec.laws.items():
        s.set_boundary_law(axis, end, rho=L.rho, velocity=L.U, pressure=L.p, rho_value=L.rho_value,
                           velocity_value=L.U_value, pressure_value=L.p_value)
    if variant is not None:
        s.variant = variant
    q = smooth_state(dim, n, seed=seed, shock=shock)
    s.upload(np.ascontiguousarray(q))
    return s, spec, q


def _initial_oracle(spec, q):
    """The oracle array the device starts from: law ends' ghost layers hold
    the boundary node (the device's extra node is uploaded that way, as the
    reference mesh initialises ghosts by clamping, SF_mesh.cpp:544); other
    ends filled by their own laws."""
    frozen = dataclasses.replace(spec, bc_lo=tuple(po.BC_FROZEN if b == po.BC_LAW else b for b in spec.bc_lo),
                                 bc_hi=tuple(po.BC_FROZEN if b == po.BC_LAW else b for b in spec.bc_hi), laws={})
    Q = spec.empty()
    spec.interior(Q)[...] = q.reshape(spec.interior(Q).shape)
    po.fill_ghosts(frozen, Q)
    ng = spec.ng
    for d in range(spec.dim):
        ax = 2 - d
        for end in (0, 1):
            if (spec.bc_hi if end else spec.bc_lo)[d] != po.BC_LAW:
                continue
            b = ng + spec.n[d] - 1 if end else ng
            plane = np.take(Q, b, axis=ax)
            for gi in (range(b + 1, b + 1 + ng) if end else range(ng)):
                idx = [slice(None)] * 4
                idx[ax] = gi
                Q[tuple(idx)] = plane
    return Q


def _kept(spec):
    """Nodes compared: not on two or more non-periodic boundary planes."""
    shape = (spec.n[2], spec.n[1], spec.n[0])
    count = np.zeros(shape, dtype=int)
    for d in range(spec.dim):
        for end in (0, 1):
            if (spec.bc_hi if end else spec.bc_lo)[d] == po.BC_PERIODIC:
                continue
            idx = [slice(None)] * 3
            idx[2 - d] = spec.n[d] - 1 if end else 0
            count[tuple(idx)] += 1
    return count < 2


CASES = {
    "1d_inflow_wall": (1, (61, 1, 1), (LAW, TR, TR), (LAW, TR, TR), {(0, 0): INFLOW, (0, 1): WALL}),
    "1d_subsonic_slip": (1, (47, 1, 1), (LAW, TR, TR), (LAW, TR, TR), {(0, 0): SUBSONIC_IN, (0, 1): SLIP}),
    "1d_outflow_transmissive": (1, (40, 1, 1), (TR, TR, TR), (LAW, TR, TR), {(0, 1): OUTFLOW}),
    "2d_channel_slip": (2, (40, 33, 1), (LAW, LAW, TR), (LAW, LAW, TR),
                        {(0, 0): INFLOW, (0, 1): OUTFLOW, (1, 0): SLIP, (1, 1): WALL}),
    "2d_periodic_y": (2, (37, 24, 1), (LAW, PER, TR), (LAW, PER, TR), {(0, 0): SUBSONIC_IN, (0, 1): SLIP}),
    "3d_duct": (3, (14, 12, 11), (LAW, LAW, PER), (LAW, TR, PER),
                {(0, 0): INFLOW, (0, 1): OUTFLOW, (1, 0): SLIP}),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_apply_boundary_matches_oracle_bitwise(case):
    dim, n, lo, hi, kinds = CASES[case]
    s, spec, q = _setup(dim, n, lo, hi, kinds, seed=3)
    Q = _initial_oracle(spec, q)
    po.fill_ghosts(spec, Q)
    s.apply_boundary()
    got = s.download().reshape(spec.interior(Q).shape)
    keep = _kept(spec)
    np.testing.assert_array_equal(got[keep], from_oracle(spec, Q)[keep])
    # the Field layout's ghosts next to each law face carry the ghost value
    ng = spec.ng
    F = s.download(layout=capi.LAYOUT_FIELD).reshape(
        tuple(spec.n[d] + 2 * ng for d in (2, 1, 0)) + (5,))
    for (axis, end) in kinds:
        ax = 2 - axis
        gi = ng + spec.n[axis] if end else ng - 1          # first ghost layer
        oi = spec.ng + spec.n[axis] if end else spec.ng - 1
        got_g = np.take(F, gi, axis=ax)
        ref_g = np.take(Q, oi, axis=ax)
        # rows of the other axes inside their solved range
        sl_f, sl_o = [], []
        for d in (2, 1, 0):
            if d == axis:
                continue
            lo_d = 1 if d < dim and (spec.bc_lo[d] != po.BC_PERIODIC) else 0
            hi_d = spec.n[d] - (1 if d < dim and spec.bc_hi[d] != po.BC_PERIODIC else 0)
            off_f = ng
            off_o = spec.ng if d < dim else 0
            sl_f.append(slice(off_f + lo_d, off_f + hi_d))
            sl_o.append(slice(off_o + lo_d, off_o + hi_d))
        np.testing.assert_array_equal(got_g[tuple(sl_f)], ref_g[tuple(sl_o)])


def _run_steps(case, recipe, time_recipe, variant, steps, precision=capi.PREC_FP64, seed=5):
    dim, n, lo, hi, kinds = CASES[case]
    s, spec, q = _setup(dim, n, lo, hi, kinds, recipe=recipe, time_recipe=time_recipe, precision=precision,
                        seed=seed, variant=variant)
    scheme, flux = split_recipe(recipe)
    Q = _initial_oracle(spec, q)
    st = po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], TIME_OF[time_recipe])
    for _ in range(steps):
        dt = po.dt(spec, Q, 0.45)
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(spec.interior(Q).shape)
    keep = _kept(spec)
    return rel_linf(got[keep], from_oracle(spec, Q)[keep]).max()


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno7Rusanov", "weno3Rusanov"])
@pytest.mark.parametrize("case", ["1d_inflow_wall", "1d_subsonic_slip", "1d_outflow_transmissive"])
def test_1d_law_steps_match_oracle(case, recipe, variant):
    assert _run_steps(case, recipe, "SSPRK3", variant, 12) <= 1e-12


@pytest.mark.parametrize("time_recipe", ["forwardEuler", "classicalRK4"])
@pytest.mark.parametrize("case", ["1d_inflow_wall", "2d_channel_slip"])
def test_law_time_recipes_match_oracle(case, time_recipe):
    assert _run_steps(case, "weno5Rusanov", time_recipe, None, 6) <= 1e-12


@pytest.mark.parametrize("variant", [0, 1, 2])
@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe"])
@pytest.mark.parametrize("case", ["2d_channel_slip", "2d_periodic_y"])
def test_2d_law_steps_match_oracle(case, recipe, variant):
    assert _run_steps(case, recipe, "SSPRK3", variant, 5) <= 1e-12


@pytest.mark.parametrize("variant", [0, 1])
def test_3d_law_steps_match_oracle(variant):
    assert _run_steps("3d_duct", "weno5Rusanov", "SSPRK3", variant, 3) <= 1e-12


@pytest.mark.parametrize("case,variant", [("1d_inflow_wall", 1), ("2d_channel_slip", 2), ("3d_duct", 1)])
def test_law_steps_fp32_flux(case, variant):
    assert _run_steps(case, "weno5Rusanov", "SSPRK3", variant, 5, precision=capi.PREC_FP32_FLUX) <= 5e-6


@pytest.mark.parametrize("case", ["1d_inflow_wall", "2d_channel_slip"])
def test_law_advance_in_graphs_matches_oracle(case):
    """sfg_advance: CFL dt, output clipping and the laws inside CUDA graphs."""
    dim, n, lo, hi, kinds = CASES[case]
    s, spec, q = _setup(dim, n, lo, hi, kinds, seed=9)
    Q = _initial_oracle(spec, q)
    t_end = 0.08
    dts, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, t_end, 0.45, write_interval=0.03)
    st, dt_gpu = s.advance(t_end, write_interval=0.03, graph_steps=8, dt_capacity=4096)
    assert st.steps == len(dts)
    np.testing.assert_allclose(dt_gpu, dts, rtol=1e-12, atol=0)
    assert abs(st.time - tf) <= 1e-12
    got = s.download().reshape(spec.interior(Q).shape)
    keep = _kept(spec)
    assert rel_linf(got[keep], from_oracle(spec, Q)[keep]).max() <= 1e-11


def test_law_changes_between_runs():
    """A law set after a graph run reaches the next run."""
    dim, n, lo, hi, kinds = CASES["1d_inflow_wall"]
    s, spec, q = _setup(dim, n, lo, hi, kinds, seed=2)
    Q = _initial_oracle(spec, q)
    po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, 0.02, 0.45)
    s.advance(0.02, graph_steps=4)
    new = po.LawSpec(*INFLOW, rho_value=1.3, U_value=(0.2, 0.0, 0.0), p_value=1.2)
    spec.laws[(0, 0)] = new
    s.set_boundary_law(0, 0, rho=new.rho, velocity=new.U, pressure=new.p, rho_value=new.rho_value,
                       velocity_value=new.U_value, pressure_value=new.p_value)
    po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, 0.04, 0.45, t_start=0.02)
    s.advance(0.04, graph_steps=4)
    got = s.download().reshape(spec.interior(Q).shape)
    assert rel_linf(got, from_oracle(spec, Q)).max() <= 1e-11
    assert got[0, 0, 0, 0] == 1.3


def test_law_arguments_are_checked():
    dim, n, lo, hi, kinds = CASES["1d_outflow_transmissive"]
    s, _, _ = _setup(dim, n, lo, hi, kinds)
    with pytest.raises(capi.SolverError):
        s.set_boundary_law(0, 0, velocity=FV)            # a transmissive end
    with pytest.raises(capi.SolverError):
        s.set_boundary_law(0, 1, velocity=7)             # unknown law
    with pytest.raises(capi.SolverError):
        s.set_boundary_law(0, 1, pressure=FV, pressure_value=0.0)
    with pytest.raises(capi.SolverError):
        s.set_boundary_law(1, 0)                         # inactive axis
    with pytest.raises(capi.SolverError):
        capi.Solver(1, (2, 1, 1), (0.5, 1, 1), (LAW, TR, TR), (TR, TR, TR))   # too few nodes
