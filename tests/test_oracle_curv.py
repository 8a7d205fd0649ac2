"""Curvilinear metrics in the oracle: per-node Jac and xi / eta / zeta
vectors, face cofactors averaged from both nodes (canonicalFace::geometry),
the residual scaled by each node's Jac, and the CFL rate from each node's
metric vectors -- pinned bit for bit to the reference operator run on a
Field holding the same metrics.  CPU only."""
import dataclasses

import numpy as np
import pytest

import pyoracle as po
from helpers import NG_OF, curvilinear_metrics, smooth_state

GRIDS = [(1, (23, 1, 1), (0.05, 1.0, 1.0)), (2, (13, 11, 1), (0.07, 0.09, 1.0)), (3, (7, 6, 5), (0.1, 0.11, 0.12))]
SCHEMES = {"weno3": po.WENO3, "weno5": po.WENO5, "teno5": po.TENO5, "weno7": po.WENO7}
FLUXES = {"Rusanov": po.RUSANOV, "Roe": po.ROE, "Steger": po.STEGER, "LaxFriedrichs": po.LAXFRIEDRICHS}


def _ref_available():
    return po.ref_lib() is not None


def curv_case(dim, n, h, scheme, bc, seed=0, shock=False):
    ng = NG_OF[scheme]
    spec = po.GridSpec(dim=dim, n=n, ng=ng, h=h, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
    spec.metrics = curvilinear_metrics(dim, n, h, ng, seed=seed)
    Q = spec.empty()
    spec.interior(Q)[...] = smooth_state(dim, n, seed=seed, shock=shock)
    po.fill_ghosts(spec, Q)
    return spec, Q


@pytest.mark.skipif(not _ref_available(), reason="reference translation units not built")
@pytest.mark.parametrize("gi", range(3))
@pytest.mark.parametrize("bc", [po.BC_TRANSMISSIVE, po.BC_PERIODIC])
def test_curvilinear_residual_and_dt_equal_reference(oracle, gi, bc):
    dim, n, h = GRIDS[gi]
    for sname in SCHEMES:
        for fname in (FLUXES if sname == "weno5" else ("Rusanov", "Roe")):
            spec, Q = curv_case(dim, n, h, sname, bc, seed=gi + 3)
            ref = po.RefCase(spec, SCHEMES[sname], FLUXES[fname])
            np.testing.assert_array_equal(po.rhs(spec, SCHEMES[sname], FLUXES[fname], Q), ref.rhs(Q),
                                          err_msg=f"{sname}{fname}")
            assert po.dt(spec, Q, 0.4) == ref.dt(Q, 0.4)


@pytest.mark.skipif(not _ref_available(), reason="reference translation units not built")
def test_curvilinear_steps_equal_reference(oracle):
    dim, n, h = GRIDS[1]
    spec, Q = curv_case(dim, n, h, "weno5", po.BC_TRANSMISSIVE, seed=7, shock=True)
    ref = po.RefCase(spec, po.WENO5, po.RUSANOV)
    mine, theirs = Q.copy(), Q.copy()
    st = po.Stepper(spec, po.WENO5, po.RUSANOV, po.SSPRK3)
    for _ in range(4):
        dt = po.dt(spec, mine, 0.4)
        st.step(mine, dt)
        ref.step(po.SSPRK3, theirs, dt)
    np.testing.assert_array_equal(mine, theirs)


@pytest.mark.parametrize("gi", range(3))
def test_cartesian_metrics_reproduce_the_uniform_path(oracle, gi):
    """Metrics of the uniform grid, given per node, give the uniform path's
    residual and dt bit for bit."""
    dim, n, h = GRIDS[gi]
    spec = po.GridSpec(dim=dim, n=n, ng=3, h=h, bc_lo=(0,) * 3, bc_hi=(0,) * 3)
    Q = spec.empty()
    spec.interior(Q)[...] = smooth_state(dim, n, seed=2)
    po.fill_ghosts(spec, Q)
    J = h[0] * h[1] * h[2]
    jac = 1.0 / J
    M = np.zeros(Q.shape[:-1] + (10,))
    M[..., 0] = jac
    M[..., 1] = (h[1] * h[2]) * jac
    M[..., 5] = (h[0] * h[2]) * jac
    M[..., 9] = (h[0] * h[1]) * jac
    curv = dataclasses.replace(spec, metrics=M)
    np.testing.assert_array_equal(po.rhs(curv, po.WENO5, po.ROE, Q), po.rhs(spec, po.WENO5, po.ROE, Q))
    assert po.dt(curv, Q, 0.5) == po.dt(spec, Q, 0.5)


def test_curvilinear_refuses_lax_wendroff(oracle):
    spec, Q = curv_case(1, (23, 1, 1), (0.05, 1.0, 1.0), "weno5", po.BC_TRANSMISSIVE)
    with pytest.raises(RuntimeError):
        po.rhs(spec, po.WENO5, po.LAXWENDROFF, Q)
