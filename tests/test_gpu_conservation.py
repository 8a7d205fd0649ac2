"""Conservation of the FP32-flux form: the conserved totals drift no more
than the FP64 path's.

Every FP32 face of a stage takes the same FP64 reference state, so a face
that two tiles, chunks or segments evaluate has the same bits in both, and
the divergence is formed from exact FP64 differences of the FP32 face
values: the fluxes telescope.  What remains is the FP64 round-off of the
stage update, the same in both precisions (SSPRK3's 1/3 and 2/3 are not
exact in binary, so both paths shed about 1e-16 of each total per step).

Measure: drift_v = (sum q_v(t) - sum q_v(0)) / sum |q_v(0)| over the nodes
(math.fsum), on periodic grids where the exact totals are constant.  Bar:
|drift_v(FP32 flux) - drift_v(FP64)| <= 1e-15 per step, summed over the
steps -- ten times the FP64 round-off scale, and far below the 1e-14 per step
that FP32 fluxes evaluated from different reference states on either side of
a tile edge leave in the momentum totals.
"""
import math

import numpy as np
import pytest

from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

PER_STEP = 1e-15


def _totals(q):
    q = q.reshape(-1, 5)
    return np.array([math.fsum(q[:, v]) for v in range(5)]), np.abs(q).sum(axis=0)


def _drift(case, precision, steps, variant=None):
    s = case.solver(precision=precision)
    if variant is not None:
        s.variant = variant
    t0, scale = _totals(s.download())
    st, _ = s.advance(1e9, max_steps=steps, graph_steps=16)
    assert st.steps == steps and st.status_bits == 0
    t1, _ = _totals(s.download())
    dev = s.totals()
    s.close()
    return (t1 - t0) / np.where(scale > 0, scale, 1.0), dev


def _periodic_tube_1d(n=3000):
    x = np.arange(n) / n
    rho = 1.0 + 0.5 * np.sin(2 * np.pi * x) + 0.3 * (np.abs(x - 0.5) < 0.15)
    u = 0.4 + 0.2 * np.cos(4 * np.pi * x)
    p = 1.0 + 0.3 * np.cos(2 * np.pi * x)
    q = cases.conserved(rho, u, 0.0, 0.0, p)[None, None]
    return cases.Case("periodic_wave_1d", 1, (n, 1, 1), (1.0 / n, 1.0, 1.0), (1, 0, 0), (1, 0, 0), q)


CASES = [
    ("vortex2d", lambda: cases.isentropic_vortex(200, recipe="teno5Rusanov"), (0, 1, 2), 300),
    ("vortex2d_roe", lambda: cases.isentropic_vortex(150, recipe="weno5Roe"), (1,), 200),
    ("taylor_green3d", lambda: cases.taylor_green(40), (0, 1), 60),
    ("wave1d", _periodic_tube_1d, (1,), 300),
]


@pytest.mark.parametrize("name,make,variants,steps", CASES, ids=[c[0] for c in CASES])
def test_fp32_flux_totals_drift_as_fp64(name, make, variants, steps):
    case = make()
    d64, _ = _drift(case, capi.PREC_FP64, steps)
    for v in variants:
        d32, dev = _drift(case, capi.PREC_FP32_FLUX, steps, variant=v)
        gap = np.abs(d32 - d64)
        assert gap.max() <= PER_STEP * steps, (name, v, d32, d64)


def test_batched_fp32_flux_totals_drift_as_fp64():
    """The persistent batch kernel over periodic vortices of uneven sizes."""
    cs = [cases.isentropic_vortex(n, recipe="weno5Rusanov", cfl=0.5) for n in (64, 90, 130)]
    steps = 200
    drifts = {}
    for prec in (capi.PREC_FP64, capi.PREC_FP32_FLUX):
        b = capi.Batch(1 << 30, 8, recipe="weno5Rusanov", precision=prec, cfl=0.5)
        slots = [b.add(c, t_end=1e9, max_steps=steps) for c in cs]
        b.step(steps + 2, graph_steps=8)
        out = []
        for c, sl in zip(cs, slots):
            t0, scale = _totals(c.q)
            t1, _ = _totals(b.download(sl))
            assert b.status(sl)["steps"] == steps
            out.append((t1 - t0) / np.where(scale > 0, scale, 1.0))
        drifts[prec] = out
        b.close()
    for d64, d32 in zip(drifts[capi.PREC_FP64], drifts[capi.PREC_FP32_FLUX]):
        assert np.abs(d32 - d64).max() <= PER_STEP * steps, (d32, d64)
