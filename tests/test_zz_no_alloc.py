"""sfg_residual_noalloc: the residual entry point for callers that cannot
allocate device memory (a host whose memory manager owns the device budget,
a fixed pre-sized memory plan, a stream that must not take cudaMalloc's
implicit device synchronisation).  It must give what sfg_residual gives.

Collected last on purpose (file name): a failure here leaves every other test
already run.  Works alone in a fresh process and after the other tests.
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import FLUX_OF, SCHEME_OF, from_oracle, oracle_spec, smooth_state, split_recipe, to_oracle
from sonicsolver_b200 import capi

pytestmark = pytest.mark.gpu

TOL = 1e-12      # the parity tolerance of the other GPU tests (FP64)
TOL_F32 = 5e-6   # FP32 fluxes: the residual tolerance of the FP32-flux tests


def _device_soa(q_nodes):
    import torch
    soa = np.ascontiguousarray(q_nodes.reshape(-1, 5).T)   # [5][nodes]
    return torch.from_numpy(soa).cuda()


def _reference_residual(dim, n, h, bc, q, recipe, precision=capi.PREC_FP64):
    s = capi.Solver(dim, n, h, (bc,) * 3, (bc,) * 3, recipe=recipe, precision=precision)
    s.upload(np.ascontiguousarray(q))
    r = s.residual().reshape(-1, 5)
    s.close()
    return r


def _oracle_residual(dim, n, h, bc, q, recipe):
    """The oracle's R = Jac * sum_d dF_d, on the solved nodes (0 elsewhere,
    as both entry points report it)."""
    spec = oracle_spec(dim, n, h, (bc,) * 3, (bc,) * 3, recipe)
    scheme, flux = split_recipe(recipe)
    R = from_oracle(spec, po.rhs(spec, SCHEME_OF[scheme], FLUX_OF[flux], to_oracle(spec, q))).reshape(q.shape)
    if bc == capi.BC_TRANSMISSIVE:
        mask = np.zeros(q.shape[:-1], bool)
        mask[(slice(1, -1) if dim > 2 else slice(None), slice(1, -1) if dim > 1 else slice(None), slice(1, -1))] = True
        R = np.where(mask[..., None], R, 0.0)
    return R.reshape(-1, 5)


def _noalloc_residual(dim, n, h, bc, q, recipe, precision=capi.PREC_FP64):
    import torch
    dq = _device_soa(q)
    dr = torch.full_like(dq, float("nan"))
    capi.residual_noalloc(dim, n, h, (bc,) * 3, (bc,) * 3, dq.data_ptr(), dr.data_ptr(), recipe=recipe,
                          precision=precision)
    torch.cuda.synchronize()
    return dr.cpu().numpy().T.copy()


def test_noalloc_matches_existing_entry_point_on_two_calls_in_a_row():
    # call 1: a larger periodic 2-D grid fills most of the shared array
    c1 = (2, (96, 80, 1), (0.02, 0.025, 1.0), capi.BC_PERIODIC, "teno5Rusanov")
    # call 2: a smaller transmissive grid; its unsolved boundary nodes must be
    # 0, not the previous call's leftovers
    c2 = (2, (37, 29, 1), (0.021, 0.017, 1.0), capi.BC_TRANSMISSIVE, "weno5Roe")
    for dim, n, h, bc, recipe in (c1, c2):
        q = smooth_state(dim, n, seed=21, shock=True)
        want = _reference_residual(dim, n, h, bc, q, recipe)
        got = _noalloc_residual(dim, n, h, bc, q, recipe)
        assert np.isfinite(got).all()
        assert rel_linf(got, want).max() <= TOL, recipe
        assert rel_linf(got, _oracle_residual(dim, n, h, bc, q, recipe)).max() <= TOL, recipe
        if bc == capi.BC_TRANSMISSIVE:
            g = got.reshape(n[1], n[0], 5)
            assert not g[0].any() and not g[-1].any() and not g[:, 0].any() and not g[:, -1].any()


@pytest.mark.parametrize("dim,n,h,bc,recipe", [
    (2, (96, 80, 1), (0.02, 0.025, 1.0), capi.BC_PERIODIC, "weno5Rusanov"),
    (3, (20, 18, 16), (0.05, 0.06, 0.07), capi.BC_TRANSMISSIVE, "teno5Roe"),
])
def test_noalloc_fp32_flux_within_fp32_tolerance(dim, n, h, bc, recipe):
    """FP32-flux mode: the sweep form of the entry point scales face fluxes by
    the area in FP64, the tile form of sfg_residual in FP32, so they agree to
    FP32 round-off (and both stay that close to the FP64 oracle); two calls
    in a row give the same bits."""
    q = smooth_state(dim, n, seed=8, shock=False)
    got = _noalloc_residual(dim, n, h, bc, q, recipe, precision=capi.PREC_FP32_FLUX)
    again = _noalloc_residual(dim, n, h, bc, q, recipe, precision=capi.PREC_FP32_FLUX)
    assert np.array_equal(got, again)
    want = _reference_residual(dim, n, h, bc, q, recipe, precision=capi.PREC_FP32_FLUX)
    assert rel_linf(got, want).max() <= TOL_F32, recipe
    assert rel_linf(got, _oracle_residual(dim, n, h, bc, q, recipe)).max() <= TOL_F32, recipe


def test_noalloc_rejects_grids_beyond_the_fixed_array():
    import torch
    n = (600, 600, 1)  # 360000 nodes > SFG_NOALLOC_MAX_NODES
    dq = torch.ones(5, 1, device="cuda", dtype=torch.float64)
    with pytest.raises(capi.SolverError) as e:
        capi.residual_noalloc(2, n, (0.01, 0.01, 1.0), (1, 1, 0), (1, 1, 0), dq.data_ptr(), dq.data_ptr())
    assert e.value.code == capi.ERR_ARG
    assert "SFG_NOALLOC_MAX_NODES" in str(e.value)
