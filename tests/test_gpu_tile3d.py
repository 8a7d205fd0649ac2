"""The fused 3-D stage kernel (variant 1: 16 x 15 columns marching up
32-plane chunks) against the oracle and against the axis sweeps.

Bars: FP64 <= 1e-12 relative L-infinity per variable per step (the parity
bar); FP32-flux <= 2e-6 (the mixed-precision step bar); FP64 variants agree
to 1e-13.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import FLUX_OF, SCHEME_OF, from_oracle, oracle_spec, smooth_state, split_recipe, to_oracle
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

GRIDS = [((14, 12, 11), (0.05, 0.06, 0.07)), ((40, 33, 70), (0.021, 0.025, 0.013)),
         ((17, 16, 33), (0.04, 0.05, 0.03))]
BCS = {"transmissive": ((0, 0, 0), (0, 0, 0)), "periodic": ((1, 1, 1), (1, 1, 1)),
       "mixed": ((capi.BC_FROZEN, 1, 0), (0, 1, capi.BC_FROZEN))}


def _oracle_state(spec, q, bc_lo, bc_hi):
    Q = spec.empty()
    spec.interior(Q)[...] = q.reshape(spec.interior(Q).shape)
    ng = spec.ng
    if bc_lo[0] == capi.BC_FROZEN:
        Q[:, :, :ng] = Q[:, :, ng:ng + 1]
    if bc_hi[2] == capi.BC_FROZEN:
        Q[-ng:] = Q[-ng - 1:-ng]
    po.fill_ghosts(spec, Q)
    return Q


def _pair(n, h, bcname, recipe, precision=capi.PREC_FP64, variant=1, seed=1, shock=True, noise=0.01):
    bc_lo, bc_hi = BCS[bcname]
    q = smooth_state(3, n, seed=seed, shock=shock, noise=noise)
    spec = oracle_spec(3, n, h, bc_lo, bc_hi, recipe)
    s = capi.Solver(3, n, h, bc_lo, bc_hi, recipe=recipe, time_recipe="SSPRK3", precision=precision, cfl=0.5)
    s.variant = variant
    s.upload(np.ascontiguousarray(q))
    return s, spec, q, _oracle_state(spec, q, bc_lo, bc_hi)


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno7Rusanov", "weno3Rusanov", "weno5Steger"])
@pytest.mark.parametrize("n,h", GRIDS)
@pytest.mark.parametrize("bcname", list(BCS))
def test_fp64_residual_matches_oracle(recipe, n, h, bcname):
    s, spec, q, Q = _pair(n, h, bcname, recipe)
    scheme, flux = split_recipe(recipe)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    bc_lo, bc_hi = BCS[bcname]
    sl = []
    for d in (2, 1, 0):   # compare on solved nodes
        a = 1 if bc_lo[d] == capi.BC_TRANSMISSIVE else 0
        b = -1 if bc_hi[d] == capi.BC_TRANSMISSIVE else None
        sl.append(slice(a, b))
    assert rel_linf(R_gpu[tuple(sl)], R_ref[tuple(sl)]).max() <= 1e-12


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Rusanov", "weno5LaxWendroff", "weno7Roe"])
@pytest.mark.parametrize("n,h", GRIDS[:2])
@pytest.mark.parametrize("bcname", list(BCS))
def test_fp64_steps_match_oracle(recipe, n, h, bcname):
    s, spec, q, Q = _pair(n, h, bcname, recipe, seed=2)
    scheme, flux = split_recipe(recipe)
    st = po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3)
    for _ in range(2):
        dt = po.dt(spec, Q, 0.5)
        assert abs(s.compute_dt() - dt) <= 1e-14 * dt
        st.step(Q, dt)
        s.step(dt)
    assert rel_linf(s.download().reshape(q.shape), from_oracle(spec, Q)).max() <= 1e-12


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Rusanov", "weno5Roe"])
@pytest.mark.parametrize("n,h", GRIDS[:2])
@pytest.mark.parametrize("bcname", ["transmissive", "periodic"])
def test_fp32_step_close_to_oracle(recipe, n, h, bcname):
    """WENO5 / Roe: the mixed-precision step bar, 2e-6 relative L-infinity.
    TENO5: its sub-stencil cut-off is a discrete decision; where FP32 flips
    one (the flip rate is measured by sfg_teno_flip_rate) that node moves by
    up to ~4e-5 relative on these shocked 3-D states -- the axis sweeps show
    the same -- so TENO5 is held to 1e-4 on the maximum and to FP32 rounding
    (1e-7) on the mean error."""
    s, spec, q, Q = _pair(n, h, bcname, recipe, precision=capi.PREC_FP32_FLUX, seed=3)
    scheme, flux = split_recipe(recipe)
    dt = po.dt(spec, Q, 0.5)
    po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3).step(Q, dt)
    s.step(dt)
    got, want = s.download().reshape(-1, 5), from_oracle(spec, Q).reshape(-1, 5)
    if recipe.startswith("teno"):
        scale = np.abs(want).max(axis=0)
        assert (np.abs(got - want).max(axis=0) / scale).max() <= 1e-4
        assert (np.abs(got - want).mean(axis=0) / scale).max() <= 1e-7
    else:
        assert rel_linf(got, want).max() <= 2e-6


def test_variants_agree_and_taylor_green_tracks_fp64():
    c = cases.taylor_green(40)
    out = {}
    for prec in (capi.PREC_FP64, capi.PREC_FP32_FLUX):
        for v in (0, 1):
            s = c.solver(precision=prec)
            s.variant = v
            st, _ = s.advance(1e30, max_steps=10, graph_steps=5)
            assert st.status_bits == 0
            out[(prec, v)] = s.download().reshape(c.q.shape)
    a, b = out[(capi.PREC_FP64, 1)].reshape(-1, 5), out[(capi.PREC_FP64, 0)].reshape(-1, 5)
    scale = np.abs(b).max(axis=0)
    scale[1:4] = scale[1:4].max()   # w starts at 0: momentum shares one scale
    assert (np.abs(a - b).max(axis=0) / scale).max() <= 1e-13
    q64, q32 = out[(capi.PREC_FP64, 1)], out[(capi.PREC_FP32_FLUX, 1)]
    ke64, ke32 = cases.kinetic_energy(q64), cases.kinetic_energy(q32)
    assert abs(ke32 - ke64) <= 1e-6 * ke64
