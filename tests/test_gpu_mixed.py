"""The FP32-flux / FP64-state path (reconstruction and face fluxes in FP32;
state, stage accumulation, totals and dt in FP64) against the FP64 oracle.

Tolerances (FP32 has a 6e-8 unit round-off):
  * one step of a smooth or shocked state: relative L-infinity per variable
    <= 2e-6 of the oracle's step (WENO3/5/7).  TENO5's cut-off is a
    threshold test, and where the FP32 indicators fall on the other side of
    it than the FP64 ones (a flip), that face's reconstruction changes by up
    to a local difference of the state: TENO5 steps are held to 1e-4 relative
    L-infinity and 1e-7 relative mean, the curvilinear FP32 tests' TENO bar;
  * a vortex run: L1(rho) error against the exact solution within 1.5x of the
    FP64 path's at the same grid and time.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import FLUX_OF, SCHEME_OF, from_oracle, oracle_spec, smooth_state, split_recipe, to_oracle
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

STEP_TOL = 2e-6
TENO_STEP_TOL, TENO_MEAN_TOL = 1e-4, 1e-7


@pytest.mark.parametrize("recipe,shock", [("weno5Rusanov", False), ("weno5Rusanov", True), ("weno5Roe", True),
                                          ("teno5Rusanov", False), ("weno3Rusanov", True), ("weno7Rusanov", False)])
@pytest.mark.parametrize("dim,n,h", [(1, (61, 1, 1), (0.013, 1.0, 1.0)), (2, (37, 29, 1), (0.021, 0.017, 1.0)),
                                     (3, (14, 12, 11), (0.05, 0.06, 0.07))])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_fp32_flux_step_close_to_fp64_oracle(recipe, shock, dim, n, h, bc):
    bcs = (bc,) * 3
    q = smooth_state(dim, n, seed=5, shock=shock)
    spec = oracle_spec(dim, n, h, bcs, bcs, recipe)
    s = capi.Solver(dim, n, h, bcs, bcs, recipe=recipe, time_recipe="SSPRK3", precision=capi.PREC_FP32_FLUX)
    s.upload(np.ascontiguousarray(q))
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    dt = po.dt(spec, Q, 0.5)
    assert abs(s.compute_dt() - dt) <= 1e-14 * dt   # dt stays FP64
    st = po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3)
    st.step(Q, dt)
    s.step(dt)
    got, want = s.download().reshape(q.shape), from_oracle(spec, Q)
    err = rel_linf(got, want)
    if scheme == "teno5":
        scale = np.abs(want).reshape(-1, 5).max(axis=0)
        mean = np.abs(got - want).reshape(-1, 5).mean(axis=0) / np.where(scale > 0, scale, 1.0)
        assert err.max() <= TENO_STEP_TOL and mean.max() <= TENO_MEAN_TOL, (err, mean)
    else:
        assert err.max() <= STEP_TOL, err


def test_fp32_vortex_l1_within_1p5x_of_fp64():
    c = cases.isentropic_vortex(64, recipe="teno5Rusanov")
    t_end = 1.0
    errs = {}
    for prec in (capi.PREC_FP64, capi.PREC_FP32_FLUX):
        s = c.solver(precision=prec)
        st, _ = s.advance(t_end)
        assert abs(st.time - t_end) < 1e-12
        q = s.download().reshape(c.q.shape)
        ex = cases.vortex_exact(c, st.time)
        errs[prec] = float(np.mean(np.abs(q[..., 0] - ex[..., 0])))
    assert errs[capi.PREC_FP32_FLUX] <= 1.5 * errs[capi.PREC_FP64], errs


def test_teno_flip_rate_diagnostic():
    """30 decisions per face; a smooth vortex flips few of them, a shocked
    state some; non-TENO recipes report none."""
    c = cases.isentropic_vortex(64, recipe="teno5Rusanov")
    s = c.solver()
    dec, flips = s.teno_flips()
    assert dec == 30 * 2 * 65 * 64   # faces f in [0, 64] per row (the wrap face counted at both ends)
    assert flips <= dec * 0.02
    q = smooth_state(2, (40, 30, 1), seed=2, shock=True)
    s2 = capi.Solver(2, (40, 30, 1), (0.02, 0.02, 1.0), (0, 0, 0), (0, 0, 0), recipe="teno5Roe")
    s2.upload(np.ascontiguousarray(q))
    d2, f2 = s2.teno_flips()
    assert d2 == 30 * ((38 + 1) * 28 + 38 * (28 + 1)) and 0 <= f2 < d2
    s3 = capi.Solver(2, (40, 30, 1), (0.02, 0.02, 1.0), (0, 0, 0), (0, 0, 0), recipe="weno5Rusanov")
    s3.upload(np.ascontiguousarray(q))
    assert s3.teno_flips() == (0, 0)


def test_fp32_vortex_far_field_has_no_nonfinite_flags():
    """Regression: near-uniform far field (smoothness indicators ~1e-26) must
    not produce 0/0 in the FP32 TENO cut-off test."""
    c = cases.isentropic_vortex(128, recipe="teno5Rusanov")
    s = c.solver(precision=capi.PREC_FP32_FLUX)
    st, _ = s.advance(1e30, max_steps=20)
    assert st.status_bits == 0 and st.steps == 20


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Rusanov", "weno5Roe"])
def test_fp32_sweep_variant_step_close_to_fp64_oracle(recipe):
    """The FP32-flux sweep kernels (2-D variant 0; the 3-D path) hold the
    stencil as FP32 deviations from one reference node per warp chunk or
    thread segment: one step within STEP_TOL of the oracle."""
    n, h, bcs = (45, 38, 1), (0.021, 0.017, 1.0), (capi.BC_PERIODIC,) * 3
    q = smooth_state(2, n, seed=9, shock=recipe != "teno5Rusanov")
    spec = oracle_spec(2, n, h, bcs, bcs, recipe)
    s = capi.Solver(2, n, h, bcs, bcs, recipe=recipe, time_recipe="SSPRK3", precision=capi.PREC_FP32_FLUX)
    s.variant = 0
    s.upload(np.ascontiguousarray(q))
    scheme, flux = split_recipe(recipe)
    Q = to_oracle(spec, q)
    dt = po.dt(spec, Q, 0.5)
    po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3).step(Q, dt)
    s.step(dt)
    got, want = s.download().reshape(q.shape), from_oracle(spec, Q)
    err = rel_linf(got, want)
    if scheme == "teno5":
        scale = np.abs(want).reshape(-1, 5).max(axis=0)
        mean = np.abs(got - want).reshape(-1, 5).mean(axis=0) / np.where(scale > 0, scale, 1.0)
        assert err.max() <= TENO_STEP_TOL and mean.max() <= TENO_MEAN_TOL, (err, mean)
    else:
        assert err.max() <= STEP_TOL, err


def test_fp32_taylor_green_tracks_fp64():
    """3-D Taylor-Green vortex (Mach 0.1, where p ~ 71 dwarfs the velocity
    variation): 20 FP32-flux steps stay within 20 x STEP_TOL of the FP64 path
    per variable, and the kinetic energy within 1e-6 relative."""
    c = cases.taylor_green(24)
    res = {}
    for prec in (capi.PREC_FP64, capi.PREC_FP32_FLUX):
        s = c.solver(precision=prec)
        st, _ = s.advance(1e30, max_steps=20, graph_steps=4)
        assert st.steps == 20 and st.status_bits == 0
        res[prec] = s.download().reshape(c.q.shape)
    q64, q32 = res[capi.PREC_FP64], res[capi.PREC_FP32_FLUX]
    assert rel_linf(q32, q64).max() <= 20 * STEP_TOL
    ke64, ke32 = cases.kinetic_energy(q64), cases.kinetic_energy(q32)
    assert abs(ke32 - ke64) <= 1e-6 * ke64
