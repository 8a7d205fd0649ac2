"""The 1-D whole-run cluster kernel (sfg_advance with 1-D kernel variant 2,
the default for 1-D grids): one thread-block cluster steps the run on device.

Against the oracle's Time::Driver loop (dt sequence and final state), and
against the graph path of variant 1, which runs the same face flux and stage
update functions (inlined into other kernels, so the compiler's contraction
of products into FMAs may differ: agreement to round-off, often bit for
bit): every recipe family, every time recipe,
transmissive / periodic / frozen ends, grids from the smallest eligible size
up, runs longer than one launch's step bound, and the cases that leave the
cluster path (too large, Lax-Wendroff, FP32 flux, boundary laws).
"""
import numpy as np
import pytest

import pyoracle as po
from conftest import rel_linf
from helpers import FLUX_OF, SCHEME_OF, TIME_OF, NG_OF, smooth_state, split_recipe
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

TR, PER, FR = capi.BC_TRANSMISSIVE, capi.BC_PERIODIC, capi.BC_FROZEN
ENDS = {"transmissive": (TR, TR), "periodic": (PER, PER), "frozen-low": (FR, TR)}


def _state(n, seed, shock):
    return np.ascontiguousarray(smooth_state(1, (n, 1, 1), seed=seed, shock=shock))


def _solver(n, ends, recipe, time_recipe, variant, q, precision=capi.PREC_FP64, h=None):
    lo, hi = ENDS[ends]
    s = capi.Solver(1, (n, 1, 1), (h or 1.0 / n, 1.0, 1.0), (lo, 0, 0), (hi, 0, 0), recipe=recipe,
                    time_recipe=time_recipe, cfl=0.5, precision=precision)
    s.variant = variant
    s.upload(q)
    return s


def _oracle_run(n, ends, recipe, time_recipe, q, steps, write_interval=0.0, t_end=1e30, h=None):
    lo, hi = ENDS[ends]
    scheme, flux = split_recipe(recipe)
    ng = NG_OF[scheme]
    spec = po.GridSpec(dim=1, n=(n, 1, 1), ng=ng, h=(h or 1.0 / n, 1.0, 1.0), bc_lo=(lo, 0, 0), bc_hi=(hi, 0, 0))
    Q = spec.empty()
    spec.interior(Q)[...] = q.reshape(spec.interior(Q).shape)
    if lo == FR:
        Q[:, :, :ng] = Q[:, :, ng:ng + 1]   # frozen low ghosts: the first node's state
    po.fill_ghosts(spec, Q)
    dts, tf = po.advance(spec, SCHEME_OF[scheme], FLUX_OF[flux], TIME_OF[time_recipe], Q, t_end, 0.5,
                         write_interval=write_interval, max_steps=steps)
    return dts, tf, np.ascontiguousarray(spec.interior(Q))


def _same(a, b, tol):
    """Round-off agreement of two dt sequences or states."""
    if tol == 0:
        np.testing.assert_array_equal(a, b)
    elif a.ndim == 1:
        np.testing.assert_allclose(a, b, rtol=tol, atol=0)
    else:
        assert rel_linf(a, b).max() <= tol


def _cluster_and_graph(n, ends, recipe, time_recipe, q, steps, **kw):
    out = []
    for v in (2, 1):
        s = _solver(n, ends, recipe, time_recipe, v, q, h=kw.get("h"))
        st, dts = s.advance(kw.get("t_end", 1e30), max_steps=steps, write_interval=kw.get("write_interval", 0.0),
                            graph_steps=16, dt_capacity=kw.get("cap", steps))
        out.append((st, dts, s.download().reshape(q.shape)))
        s.close()
    return out


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno3Rusanov", "weno7Rusanov", "weno5Steger",
                                    "teno5LaxFriedrichs"])
@pytest.mark.parametrize("time_recipe", ["forwardEuler", "SSPRK3", "classicalRK4"])
@pytest.mark.parametrize("ends", list(ENDS))
def test_cluster_run_matches_oracle_and_graph_path(recipe, time_recipe, ends):
    n = 203
    euler = time_recipe == "forwardEuler"
    steps = 12 if euler else 40
    q = _state(n, seed=7, shock=not euler)
    (st2, dts2, q2), (st1, dts1, q1) = _cluster_and_graph(n, ends, recipe, time_recipe, q, steps)
    # the graph path (same face flux and stage functions)
    assert st2.steps == st1.steps == steps
    _same(dts2, dts1, 1e-11)
    _same(q2, q1, 1e-10)
    assert abs(st2.time - st1.time) <= 1e-14
    # and the oracle's time loop
    dts_ref, tf, ref = _oracle_run(n, ends, recipe, time_recipe, q, steps)
    assert len(dts_ref) == steps
    np.testing.assert_allclose(dts2, dts_ref, rtol=1e-11, atol=0)
    assert abs(st2.time - tf) <= 1e-13 * max(1.0, abs(tf))
    sl = slice(1, -1) if ends == "transmissive" else slice(None)
    assert rel_linf(q2[:, :, sl], ref.reshape(q.shape)[:, :, sl]).max() <= 1e-10


@pytest.mark.parametrize("n,ends", [(10, "transmissive"), (11, "periodic"), (12, "frozen-low"), (17, "transmissive"),
                                    (65, "periodic"), (2049, "transmissive"), (8192, "periodic")])
def test_grid_sizes_split_over_the_cluster(n, ends):
    """From the smallest eligible grid (8 solved nodes: one per CTA, trailing
    CTAs idle for the shorter chunks) to the largest (8192 nodes)."""
    q = _state(n, seed=3, shock=True)
    steps = 20
    (st2, dts2, q2), (st1, dts1, q1) = _cluster_and_graph(n, ends, "weno5Rusanov", "SSPRK3", q, steps)
    _same(dts2, dts1, 1e-11)
    _same(q2, q1, 1e-10)
    dts_ref, _, ref = _oracle_run(n, ends, "weno5Rusanov", "SSPRK3", q, steps)
    np.testing.assert_allclose(dts2, dts_ref, rtol=1e-11, atol=0)
    sl = slice(1, -1) if ends == "transmissive" else slice(None)
    assert rel_linf(q2[:, :, sl], ref.reshape(q.shape)[:, :, sl]).max() <= 1e-10


def test_sod_run_to_end_time_with_output_clipping():
    """The 1000-cell Sod run to t = 0.2 with output times every 0.05: the
    cluster clips dt at the output times and the end exactly as the graph
    path and the oracle's loop."""
    c = cases.sod_1d(1000)
    q = np.ascontiguousarray(c.q)
    n = c.n[0]   # 1001 nodes: 1000 cells between them
    (st2, dts2, q2), (st1, dts1, q1) = _cluster_and_graph(n, "transmissive", "weno5Rusanov", "SSPRK3", q, 0,
                                                          t_end=c.t_end, write_interval=0.05, cap=4000, h=c.h[0])
    assert st2.steps == st1.steps > 800
    _same(dts2, dts1, 1e-11)
    _same(q2, q1, 1e-10)
    assert abs(st2.time - st1.time) <= 1e-15
    dts_ref, tf, ref = _oracle_run(n, "transmissive", "weno5Rusanov", "SSPRK3", q, 10 ** 6,
                                   write_interval=0.05, t_end=c.t_end, h=c.h[0])
    assert st2.steps == len(dts_ref)
    np.testing.assert_allclose(dts2, dts_ref, rtol=1e-11, atol=0)
    assert abs(st2.time - tf) <= 1e-14
    assert rel_linf(q2[:, :, 1:-1], ref.reshape(q.shape)[:, :, 1:-1]).max() <= 1e-10


def test_run_longer_than_one_launch():
    """5000 steps: the kernel stops after 4096 and the host launches it again
    from the clock it left."""
    n = 64
    q = _state(n, seed=11, shock=False)
    (st2, dts2, q2), (st1, dts1, q1) = _cluster_and_graph(n, "periodic", "weno5Rusanov", "SSPRK3", q, 5000)
    assert st2.steps == st1.steps == 5000
    _same(dts2, dts1, 1e-11)
    _same(q2, q1, 1e-11)


def test_repeated_advances_continue_the_clock():
    n = 300
    q = _state(n, seed=2, shock=True)
    res = []
    for v in (2, 1):
        s = _solver(n, "transmissive", "teno5Rusanov", "SSPRK3", v, q)
        for _ in range(3):
            s.advance(1e30, max_steps=7, graph_steps=4)
        res.append((s.time(), s.download()))
        s.close()
    assert res[0][0][1] == res[1][0][1] == 21
    assert abs(res[0][0][0] - res[1][0][0]) <= 1e-15
    _same(res[0][1].reshape(-1, 5), res[1][1].reshape(-1, 5), 1e-13)


@pytest.mark.parametrize("what", ["too_large", "lax_wendroff", "fp32_flux"])
def test_ineligible_grids_take_the_graph_path(what):
    n = 9000 if what == "too_large" else 301
    recipe = "weno5LaxWendroff" if what == "lax_wendroff" else "weno5Rusanov"
    prec = capi.PREC_FP32_FLUX if what == "fp32_flux" else capi.PREC_FP64
    q = _state(n, seed=5, shock=False)
    out = []
    for v in (2, 1):
        s = _solver(n, "periodic", recipe, "SSPRK3", v, q, precision=prec)
        st, _ = s.advance(1e30, max_steps=6, graph_steps=3)
        assert st.steps == 6
        out.append(s.download())
        s.close()
    np.testing.assert_array_equal(out[0], out[1])


def test_invalid_state_stops_the_run_with_an_error():
    n = 120
    q = _state(n, seed=1, shock=False)
    bad = q.copy()
    bad[0, 0, 60, 4] = -1.0   # negative total energy: p < 0
    s = _solver(n, "transmissive", "weno5Rusanov", "SSPRK3", 2, np.ascontiguousarray(bad))
    with pytest.raises(capi.SolverError) as e:
        s.advance(1e30, max_steps=10)
    assert e.value.code == capi.ERR_STATE
    assert s.status() != 0


def test_default_variant_by_dimension():
    s = _solver(61, "periodic", "weno5Rusanov", "SSPRK3", 2, _state(61, 0, False))
    s.variant = 0
    s.variant = 1
    s.variant = 2
    c = capi.Solver(1, (61, 1, 1), (0.01, 1.0, 1.0), (PER, 0, 0), (PER, 0, 0))
    assert c.variant == 2


@pytest.mark.parametrize("dim", [1, 2])
def test_max_dt_clips_every_step_like_the_oracle(dim):
    """numerics maxDeltaT (FlowDtCompute's min with the CFL dt): 1-D runs in
    the cluster kernel, 2-D in the graph path; a dt log shorter than the run
    keeps the first steps."""
    n = (120, 1, 1) if dim == 1 else (40, 36, 1)
    h = (1.0 / n[0], 1.0 / max(n[1], 1), 1.0)
    bc = (TR, TR if dim > 1 else 0, 0)
    q = np.ascontiguousarray(smooth_state(dim, n, seed=9, shock=True))
    spec = po.GridSpec(dim=dim, n=n, ng=3, h=h, bc_lo=bc, bc_hi=bc)
    Q = spec.empty()
    spec.interior(Q)[...] = q.reshape(spec.interior(Q).shape)
    po.fill_ghosts(spec, Q)
    free_dt = po.dt(spec, Q, 0.5)
    max_dt = 0.6 * free_dt
    dts_ref, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, 1e30, 0.5, max_dt=max_dt, max_steps=20)
    s = capi.Solver(dim, n, h, bc, bc, recipe="weno5Rusanov", cfl=0.5, max_dt=max_dt)
    s.upload(q)
    st, dts = s.advance(1e30, max_steps=20, graph_steps=8, dt_capacity=5)
    assert st.steps == 20 and len(dts) == 5
    assert (dts_ref <= max_dt).all() and (dts_ref == max_dt).any()
    np.testing.assert_allclose(dts, dts_ref[:5], rtol=1e-12, atol=0)
    assert abs(st.time - tf) <= 1e-14
    sl = (slice(None),) * (3 - dim) + (slice(1, -1),) * dim
    got = s.download().reshape(q.shape)
    ref = np.ascontiguousarray(spec.interior(Q)).reshape(q.shape)
    assert rel_linf(got[sl], ref[sl]).max() <= 1e-11
