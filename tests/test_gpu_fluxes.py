"""Steger-Warming, Lax-Friedrichs and Lax-Wendroff faces on the GPU (FP64)
against the oracle, whose restatement of the three fluxes is pinned bit for
bit to the reference translation units (tests/test_oracle.py).

Bar: <= 1e-12 relative L-infinity per conserved variable per step, as the
other parity tests.  Lax-Wendroff uses the step's dt, so it is compared at
step level.
"""
import os
import json
import subprocess

import numpy as np
import pytest

import pyoracle as po
from case_dirs import write_case
from conftest import rel_linf
from helpers import FLUX_OF, SCHEME_OF, from_oracle, oracle_spec, smooth_state, split_recipe, to_oracle
from sonicsolver_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-12
GRIDS = [
    (1, (61, 1, 1), (0.013, 1.0, 1.0)),
    (2, (37, 29, 1), (0.021, 0.017, 1.0)),
    (3, (14, 12, 11), (0.05, 0.06, 0.07)),
]
SCHEMES = ["weno3", "weno5", "teno5", "weno7"]


def _solver(dim, n, h, bc, recipe, time_recipe="SSPRK3", variant=None, seed=0):
    bcs = (bc,) * 3
    q = smooth_state(dim, n, seed=seed, shock=True)
    spec = oracle_spec(dim, n, h, bcs, bcs, recipe)
    s = capi.Solver(dim, n, h, bcs, bcs, recipe=recipe, time_recipe=time_recipe, cfl=0.5)
    if variant is not None:
        s.variant = variant
    s.upload(np.ascontiguousarray(q))
    return s, spec, q


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("flux", ["Steger", "LaxFriedrichs"])
@pytest.mark.parametrize("dim,n,h", GRIDS)
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_residual_parity(scheme, flux, dim, n, h, bc):
    recipe = scheme + flux
    s, spec, q = _solver(dim, n, h, bc, recipe)
    Q = to_oracle(spec, q)
    R_ref = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], Q))
    R_gpu = s.residual().reshape(R_ref.shape)
    sl = tuple(slice(1, -1) if (d < dim and bc == capi.BC_TRANSMISSIVE) else slice(None) for d in (2, 1, 0))
    assert rel_linf(R_gpu[sl], R_ref[sl]).max() <= TOL


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("flux", ["Steger", "LaxFriedrichs", "LaxWendroff"])
@pytest.mark.parametrize("dim,n,h,variant", [(1, (61, 1, 1), (0.013, 1.0, 1.0), 1),
                                             (2, (37, 29, 1), (0.021, 0.017, 1.0), 1),
                                             (2, (37, 29, 1), (0.021, 0.017, 1.0), 0),
                                             (3, (14, 12, 11), (0.05, 0.06, 0.07), 0)])
@pytest.mark.parametrize("bc", [capi.BC_TRANSMISSIVE, capi.BC_PERIODIC])
def test_step_parity(scheme, flux, dim, n, h, variant, bc):
    """Two SSPRK3 steps at the oracle's CFL dt: 1-D tile, 2-D tile and sweep,
    3-D sweeps."""
    recipe = scheme + flux
    s, spec, q = _solver(dim, n, h, bc, recipe, variant=variant, seed=3)
    Q = to_oracle(spec, q)
    st = po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3)
    for _ in range(2):
        dt = po.dt(spec, Q, 0.5)
        assert abs(s.compute_dt() - dt) <= 1e-14 * dt
        st.step(Q, dt)
        s.step(dt)
    err = rel_linf(s.download().reshape(q.shape), from_oracle(spec, Q))
    assert err.max() <= TOL, err


@pytest.mark.parametrize("recipe", ["weno5Steger", "teno5LaxFriedrichs", "weno5LaxWendroff"])
def test_fp32_flux_mode_and_batches_refuse_these_faces(recipe):
    with pytest.raises(capi.SolverError) as e:
        capi.Solver(1, (40, 1, 1), (0.02, 1.0, 1.0), (0, 0, 0), (0, 0, 0), recipe=recipe,
                    precision=capi.PREC_FP32_FLUX)
    assert e.value.code == capi.ERR_ARG and "Rusanov and Roe" in str(e.value)
    with pytest.raises(capi.SolverError):
        capi.Batch(1 << 24, 4, recipe=recipe)


def test_steger_frozen_sod_case_through_the_plan(tmp_path):
    """A case directory shaped like the reference's sodCase (TENO5 +
    Steger-Warming, forwardEuler, no Left condition) through sfg_run, against
    the oracle's run of the same case."""
    nx, ny = 101, 11
    d = write_case(str(tmp_path), "sod_sw", cells=(nx - 1, ny - 1, 1), box_hi=(100.0, 10.0, 0.1), n_ghost=3,
                   convection="teno5StegerWarming", numerics_form="scheme", time="forwardEuler", end_time=0.02,
                   cfl=0.5, write_interval=0.01, left=(1.0, 0.0, 1e5), right=(0.125, 0.0, 1e4),
                   boundaries={"Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"})
    out = os.path.join(d, "final.bin")
    runner = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "sonicsolver_b200", "sfg_run")
    r = subprocess.run([runner, d, "--no-write", "--dump", out], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    summary = json.loads(r.stdout.strip().splitlines()[-1])
    assert summary["recipe"] == "teno5Steger" and "bc=20/00/00" in r.stdout
    spec = po.GridSpec(dim=2, n=(nx, ny, 1), ng=3, h=(1.0, 1.0, 0.1), bc_lo=(po.BC_FROZEN, po.BC_TRANSMISSIVE, 0),
                       bc_hi=(po.BC_TRANSMISSIVE, po.BC_TRANSMISSIVE, 0))
    Q = spec.empty()
    I = spec.interior(Q)
    left = np.arange(nx) < nx // 2
    I[..., 0] = np.where(left, 1.0, 0.125)
    I[..., 4] = np.where(left, 1e5, 1e4) / 0.4
    Q[:, :, :3] = Q[:, :, 3:4]   # frozen ghosts: the initial clamp
    po.fill_ghosts(spec, Q)
    dts, tf = po.advance(spec, po.TENO5, po.STEGER, po.EULER, Q, 0.02, 0.5, write_interval=0.01)
    assert summary["steps"] == len(dts) and abs(summary["time"] - tf) <= 1e-15
    got = np.fromfile(out).reshape(-1, 5)
    assert rel_linf(got, np.ascontiguousarray(spec.interior(Q)).reshape(-1, 5)).max() <= 1e-11
