"""Pins the CPU oracle (oracle/sf_oracle.c) before it is trusted as the checker.

1. Known-answer tests of the reference's own suite:
   test/test_numericalFlux.cpp:106-233 (constant-state preservation, flux
   consistency, distinct fluxes) and test/test_explicitStages.cpp:95-160
   (stage coefficients, stage times, constant-RHS final value 9.8).
2. Bit-for-bit agreement with the reference translation units compiled in
   place (oracle/_ref) on seeded states, and with the committed fixtures
   tests/golden/ref_rhs.npz generated from them.
3. The frozen WENO7 + Rusanov + forwardEuler Sod baseline
   (test/Sod/sodCase_weno7_t0p2/baseline.json -> tests/golden/sod_weno7_t0p2.json).
"""
import ctypes
import json
import os

import numpy as np
import pytest

import pyoracle as po
from helpers import NG_OF, smooth_state

HERE = os.path.dirname(os.path.abspath(__file__))
GAMMA = 1.4


def near(a, b, tol=1e-12):
    return abs(a - b) <= tol * max(1.0, abs(a), abs(b))


def perfect_gas_state(rho, u, v, w, p, gamma=GAMMA):
    return np.array([rho, rho * u, rho * v, rho * w, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)])


def dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


UNIFORM = perfect_gas_state(1.2, 30.0, -2.0, 1.0, 101325.0)
PHYS_UNIFORM = np.array([UNIFORM[1], UNIFORM[1] * 30.0 + 101325.0, UNIFORM[2] * 30.0, UNIFORM[3] * 30.0,
                         (UNIFORM[4] + 101325.0) * 30.0])


# ---------------------------------------------------------------- 1. KATs

@pytest.mark.parametrize("scheme,nst", [(po.WENO3, 4), (po.WENO5, 6), (po.TENO5, 6), (po.WENO7, 8)])
def test_constant_state_preserved(oracle, scheme, nst):
    """reconstructedConstantState: L, R inverse and every core exact on a
    constant stencil (test_numericalFlux.cpp:44-93)."""
    lib = po.oracle_lib()
    n = np.array([1.0, 0.0, 0.0])
    L = np.zeros(25)
    R = np.zeros(25)
    assert lib.sfo_char_matrix(dp(UNIFORM), dp(n), GAMMA, dp(L), dp(R)) == 0
    L, R = L.reshape(5, 5), R.reshape(5, 5)
    w = L @ UNIFORM
    width = {4: 4, 6: 5, 8: 7}[nst]
    core = {po.WENO3: lib.sfo_weno3_core, po.WENO5: lib.sfo_weno5_core, po.WENO7: lib.sfo_weno7_core}.get(scheme)
    rec = np.zeros(5)
    for v in range(5):
        st = np.full(8, w[v])
        rec[v] = po.oracle_lib().sfo_teno5_core(dp(st), None) if scheme == po.TENO5 else core(dp(st))
    q = R @ rec
    assert all(near(q[v], UNIFORM[v]) for v in range(5))
    _ = width


def test_rusanov_uniform_equals_physical_flux(oracle):
    out = np.zeros(5)
    n = np.array([1.0, 0.0, 0.0])
    assert po.oracle_lib().sfo_rusanov_flux(dp(UNIFORM), dp(UNIFORM), dp(n), GAMMA, dp(out)) == 0
    assert all(near(out[v], PHYS_UNIFORM[v]) for v in range(5))


def test_roe_uniform_equals_physical_flux(oracle):
    out = np.zeros(5)
    n = np.array([1.0, 0.0, 0.0])
    assert po.oracle_lib().sfo_roe_flux(dp(UNIFORM), dp(UNIFORM), dp(n), GAMMA, dp(out)) == 0
    assert all(near(out[v], PHYS_UNIFORM[v]) for v in range(5))


@pytest.mark.parametrize("flux", [po.RUSANOV, po.ROE])
def test_reconstructed_flux_consistent_on_constant_stencil(oracle, flux):
    """reconstructedConstantFlux with metrics {1,0,0,1} (test_numericalFlux.cpp:96-104,144-158)."""
    st = np.tile(UNIFORM, 6)
    metrics = np.array([1.0, 0.0, 0.0, 1.0])
    out = np.zeros(5)
    assert po.oracle_lib().sfo_char_face_flux(6, dp(st), dp(metrics), po.WENO5, flux, GAMMA, dp(out)) == 0
    assert all(near(out[v], PHYS_UNIFORM[v]) for v in range(5))


def test_fluxes_distinct_on_riemann_data(oracle):
    """Configured fluxes are observably distinct (test_numericalFlux.cpp:160-175)."""
    left = perfect_gas_state(1.0, 2.0, 0.1, 0.0, 1.0)
    right = perfect_gas_state(0.125, -0.5, 0.0, 0.0, 0.1)
    n = np.array([1.0, 0.0, 0.0])
    rus, roe = np.zeros(5), np.zeros(5)
    po.oracle_lib().sfo_rusanov_flux(dp(left), dp(right), dp(n), GAMMA, dp(rus))
    po.oracle_lib().sfo_roe_flux(dp(left), dp(right), dp(n), GAMMA, dp(roe))
    assert not all(near(rus[v], roe[v], 1e-10) for v in range(5))


SSP = [(0.0, 0.0, 1.0), (1.0, 0.75, 0.25), (0.5, 1.0 / 3.0, 2.0 / 3.0)]
RK4 = [(0.0, 0.0, 0.5), (0.5, 0.0, 0.5), (0.5, 0.0, 1.0), (1.0, 0.0, 0.0)]


@pytest.mark.parametrize("time_id,stage_times", [(po.EULER, [2.0]), (po.SSPRK3, [2.0, 2.1, 2.05]),
                                                 (po.RK4, [2.0, 2.05, 2.05, 2.1])])
def test_constant_rhs_stage_math(oracle, time_id, stage_times):
    """runConstantRhs (test_explicitStages.cpp:39-84): source -2 on E at t=2,
    dt=0.1 -> E = 9.8 to 1e-14 for Euler, SSPRK3 and RK4; stage times from
    the tableaux abscissae."""
    lib = po.oracle_lib()
    spec = po.GridSpec(dim=1, n=(3, 1, 1), ng=3, bc_lo=(po.BC_PERIODIC,) * 3, bc_hi=(po.BC_PERIODIC,) * 3)
    Q = spec.empty()
    spec.interior(Q)[..., 0] = 1.0
    spec.interior(Q)[..., 4] = 10.0
    calls = []

    @po.ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))
    def const_rhs(ctx, q, r):
        calls.append(1)
        size = Q.size
        arr = np.ctypeslib.as_array(r, shape=(size,))
        arr[:] = 0.0
        arr[4::5] = 2.0   # R = Jac*div - source = 0 - (-2)
        return 0

    lib.sfo_stage_fn.argtypes = [ctypes.POINTER(po.Grid), ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_double), ctypes.c_double, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_double)]
    g = spec.c()
    work = np.zeros(5 * Q.size)
    stages = len(stage_times)
    t, dt = 2.0, 0.1
    tableau = {po.EULER: [(0.0, 0.0, 1.0)], po.SSPRK3: SSP, po.RK4: RK4}[time_id]
    for s in range(stages):
        assert abs(t + tableau[s][0] * dt - stage_times[s]) < 1e-14
        assert lib.sfo_stage_fn(ctypes.byref(g), ctypes.cast(const_rhs, ctypes.c_void_p), None, time_id, dp(Q), dt,
                                s, dp(work)) == 0
    assert len(calls) == stages
    assert np.all(np.abs(spec.interior(Q)[..., 4] - 9.8) < 1e-14)


# ---------------------------------------------------------------- 2. vs reference TUs

def _ref_available():
    return po.ref_lib() is not None


GRIDS = [(1, (23, 1, 1), (0.05, 1.0, 1.0)), (2, (13, 11, 1), (0.07, 0.09, 1.0)), (3, (7, 6, 5), (0.1, 0.11, 0.12))]
RECIPES = [("weno5", "Rusanov"), ("weno5", "Roe"), ("teno5", "Rusanov"), ("teno5", "Roe"), ("weno3", "Rusanov"),
           ("weno7", "Rusanov")]
SCHEMES = {"weno3": po.WENO3, "weno5": po.WENO5, "teno5": po.TENO5, "weno7": po.WENO7}
FLUXES = {"Rusanov": po.RUSANOV, "Roe": po.ROE}


def test_oracle_matches_committed_reference_fixtures(oracle):
    """Bit-for-bit against the reference operator's outputs in ref_rhs.npz."""
    data = np.load(os.path.join(HERE, "golden", "ref_rhs.npz"))
    checked = 0
    for gi, (dim, n, _h) in enumerate(GRIDS):
        for bc in (po.BC_TRANSMISSIVE, po.BC_PERIODIC):
            for shock in ((True,) if dim == 3 else (False, True)):
                state = f"{dim}d_bc{bc}_{'shock' if shock else 'smooth'}"
                q, h = data[state + "_q"], tuple(data[state + "_h"])
                for sname, fname in RECIPES:
                    spec = po.GridSpec(dim=dim, n=n, ng=NG_OF[sname], h=h, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
                    Q = spec.empty()
                    spec.interior(Q)[...] = q
                    po.fill_ghosts(spec, Q)
                    R = spec.interior(po.rhs(spec, SCHEMES[sname], FLUXES[fname], Q))
                    np.testing.assert_array_equal(R, data[f"{state}_{sname}{fname}_r"])
                    checked += 1
    assert checked == 6 * (2 * 2 + 2 * 2 + 2)


@pytest.mark.skipif(not _ref_available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("sname,fname", RECIPES)
def test_oracle_bitwise_equals_reference_operator(oracle, sname, fname):
    for gi, (dim, n, h) in enumerate(GRIDS):
        for bc in (po.BC_TRANSMISSIVE, po.BC_PERIODIC):
            q = smooth_state(dim, n, seed=100 + gi, shock=True)
            spec = po.GridSpec(dim=dim, n=n, ng=NG_OF[sname], h=h, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
            Q = spec.empty()
            spec.interior(Q)[...] = q
            po.fill_ghosts(spec, Q)
            rc = po.RefCase(spec, SCHEMES[sname], FLUXES[fname])
            np.testing.assert_array_equal(po.rhs(spec, SCHEMES[sname], FLUXES[fname], Q), rc.rhs(Q))
            assert po.dt(spec, Q, 0.5) == rc.dt(Q, 0.5)


@pytest.mark.skipif(not _ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_oracle_time_loop_equals_reference_operator_loop(oracle):
    """The whole Time::Driver loop around the reference operator vs around the
    restatement: identical dt sequence and state (SSPRK3, TENO5, Sod)."""
    spec = po.GridSpec(dim=1, n=(101, 1, 1), ng=3, h=(0.01, 1.0, 1.0))
    Q = spec.empty()
    x = np.arange(101) * 0.01
    I = spec.interior(Q)
    I[..., 0] = np.where(x < 0.5, 1.0, 0.125)
    I[..., 4] = np.where(x < 0.5, 1.0, 0.1) / 0.4
    Q2 = Q.copy()
    d1, t1 = po.advance(spec, po.TENO5, po.RUSANOV, po.SSPRK3, Q, 0.05, 0.5)
    d2, t2 = po.RefCase(spec, po.TENO5, po.RUSANOV).advance(po.SSPRK3, Q2, 0.05, 0.5)
    np.testing.assert_array_equal(d1, d2)
    np.testing.assert_array_equal(Q, Q2)


# ---------------------------------------------------------------- 3. Sod golden

def _sod_run():
    with open(os.path.join(HERE, "golden", "sod_weno7_t0p2.json")) as f:
        fx = json.load(f)
    c = fx["case"]
    nx, ny, _ = c["nodes"]
    ng = c["n_ghost"]
    spec = po.GridSpec(dim=2, n=(nx, ny, 1), ng=ng, h=(1.0, 1.0, 0.1), bc_lo=(po.BC_FROZEN, po.BC_TRANSMISSIVE, 0),
                       bc_hi=(po.BC_TRANSMISSIVE, po.BC_TRANSMISSIVE, 0))
    Q = spec.empty()
    I = spec.interior(Q)
    for i in range(nx):
        s = c["left"] if i < c["split_node"] else c["right"]
        I[:, :, i, 0] = s["rho"]
        I[:, :, i, 4] = s["p"] / (c["gamma"] - 1.0)
    # initializeGhostStateFromInterior (SF_mesh.cpp:544): ghosts clamp to the interior
    Q[:, :, :ng] = Q[:, :, ng:ng + 1]
    Q[:, :, ng + nx:] = Q[:, :, ng + nx - 1:ng + nx]
    Q[:, :ng] = Q[:, ng:ng + 1]
    Q[:, ng + ny:] = Q[:, ng + ny - 1:ng + ny]
    dts, tf = po.advance(spec, po.WENO7, po.RUSANOV, po.EULER, Q, c["t_end"], c["cfl"],
                         write_interval=c["write_interval"])
    return fx["baseline"], spec, Q, dts, tf


@pytest.fixture(scope="module")
def sod_run(oracle):
    return _sod_run()


def test_sod_golden_steps_and_dt_sequence(sod_run):
    base, spec, Q, dts, tf = sod_run
    assert len(dts) == base["steps"] == 454
    assert abs(tf - base["final_time"]) <= 5e-12
    # first dt to all digits of the reference's trace (6.681531047810609e-4)
    assert abs(dts[0] - 6.681531047810609e-4) <= 1e-18
    # the log prints dt with 7 significant digits.  The first 300 steps round
    # alike digit for digit; later steps drift with the case's sensitivity
    # (the final clip dt = 0.2 - t carries the accumulated time difference),
    # all within 1e-6 relative.
    for i, (got, exp) in enumerate(zip(dts, base["dt_sequence"])):
        if i < 300:
            assert float(f"{got:.6e}") == pytest.approx(exp, rel=5e-12, abs=0), i
        assert abs(got - exp) <= 1e-6 * exp, i


def _integrals(spec, Q, gamma=GAMMA):
    I = spec.interior(Q)[0]
    rho = I[..., 0]
    u, v, w = I[..., 1] / rho, I[..., 2] / rho, I[..., 3] / rho
    p = (gamma - 1.0) * (I[..., 4] - 0.5 * rho * (u * u + v * v + w * w))
    W = np.ones(rho.shape)
    W[:, 0] *= 0.5
    W[:, -1] *= 0.5
    W[0, :] *= 0.5
    W[-1, :] *= 0.5
    W *= 0.5 * 0.1 * 2   # 2 z-nodes in the reference mesh, trapezoid weight 0.5 each
    return {"rho": (rho.min(), rho.max()), "p": (p.min(), p.max()),
            "speed": (np.sqrt(u * u + v * v + w * w).min(), np.sqrt(u * u + v * v + w * w).max()),
            "mass": (W * rho).sum(), "momentum": [(W * I[..., k]).sum() for k in (1, 2, 3)],
            "energy": (W * I[..., 4]).sum()}


def test_sod_golden_ranges_and_integrals(sod_run):
    """The reference's checker compares at 5e-12, but this case amplifies a
    1e-15 perturbation of one node to ~1e-10 in mass (see the sensitivity test
    below), so only a run that repeats every rounding of the original build
    meets it.  Bars here: 2e-10 on integrals, 2e-7 on ranges, and the
    y-momentum (pure metric round-off in the reference) below 1e-7."""
    base, spec, Q, dts, tf = sod_run
    got = _integrals(spec, Q)
    for k in ("rho", "p", "speed"):
        for a, b in zip(got[k], base["ranges"][k]):
            assert abs(a - b) <= 2e-7 * abs(b), (k, a, b)
    assert abs(got["mass"] - base["integrals"]["mass"]) <= 2e-10 * base["integrals"]["mass"]
    assert abs(got["energy"] - base["integrals"]["energy"]) <= 2e-10 * base["integrals"]["energy"]
    mx = base["integrals"]["momentum"][0]
    assert abs(got["momentum"][0] - mx) <= 2e-10 * mx
    assert abs(got["momentum"][1]) < 1e-7 and abs(base["integrals"]["momentum"][1]) < 1e-7
    assert got["momentum"][2] == base["integrals"]["momentum"][2] == 0.0


def test_sod_golden_sensitivity_bounds_the_bar(sod_run):
    """A 1e-15 relative change of one node's energy moves the final mass by
    more than 1e-11 relative: the golden cannot pin below that level."""
    base, spec, Q, dts, tf = sod_run
    with open(os.path.join(HERE, "golden", "sod_weno7_t0p2.json")) as f:
        c = json.load(f)["case"]
    m0 = _integrals(spec, Q)["mass"]
    _, spec2, Q2, _, _ = _sod_perturbed(c)
    m1 = _integrals(spec2, Q2)["mass"]
    assert abs(m1 - m0) / m0 > 1e-11


def _sod_perturbed(c):
    nx, ny, _ = c["nodes"]
    ng = c["n_ghost"]
    spec = po.GridSpec(dim=2, n=(nx, ny, 1), ng=ng, h=(1.0, 1.0, 0.1), bc_lo=(po.BC_FROZEN, po.BC_TRANSMISSIVE, 0),
                       bc_hi=(po.BC_TRANSMISSIVE, po.BC_TRANSMISSIVE, 0))
    Q = spec.empty()
    I = spec.interior(Q)
    for i in range(nx):
        s = c["left"] if i < c["split_node"] else c["right"]
        I[:, :, i, 0] = s["rho"]
        I[:, :, i, 4] = s["p"] / (c["gamma"] - 1.0)
    I[0, 10, 60, 4] *= 1.0 + 1e-15
    Q[:, :, :ng] = Q[:, :, ng:ng + 1]
    Q[:, :, ng + nx:] = Q[:, :, ng + nx - 1:ng + nx]
    Q[:, :ng] = Q[:, ng:ng + 1]
    Q[:, ng + ny:] = Q[:, ng + ny - 1:ng + ny]
    dts, tf = po.advance(spec, po.WENO7, po.RUSANOV, po.EULER, Q, c["t_end"], c["cfl"],
                         write_interval=c["write_interval"])
    return None, spec, Q, dts, tf


# ------------------------------------- 4. Steger-Warming, Lax-Friedrichs, Lax-Wendroff

NEW_FLUXES = {"Steger": po.STEGER, "LaxFriedrichs": po.LAXFRIEDRICHS, "LaxWendroff": po.LAXWENDROFF}


def _flux(name, qL, qR, n, dt=1e-3, spacing=0.1):
    out = np.zeros(5)
    lib = po.oracle_lib()
    if name == "Steger":
        rc = lib.sfo_steger_flux(dp(qL), dp(qR), dp(n), GAMMA, dp(out))
    elif name == "LaxFriedrichs":
        rc = lib.sfo_lf_flux(dp(qL), dp(qR), dp(n), GAMMA, dp(out))
    else:
        rc = lib.sfo_lw_flux(dp(qL), dp(qR), dp(n), dt, spacing, GAMMA, dp(out))
    assert rc == 0
    return out


@pytest.mark.parametrize("name", list(NEW_FLUXES))
def test_new_fluxes_uniform_equal_physical_flux(oracle, name):
    """Equal-state fluxes reduce to the physical flux (test_numericalFlux.cpp:185-199)."""
    out = _flux(name, UNIFORM, UNIFORM, np.array([1.0, 0.0, 0.0]))
    assert all(near(out[v], PHYS_UNIFORM[v]) for v in range(5))


@pytest.mark.parametrize("name", ["Steger", "LaxFriedrichs"])
def test_new_fluxes_reconstructed_on_constant_stencil(oracle, name):
    """reconstructedConstantFlux with SW / LF (test_numericalFlux.cpp:201-224)."""
    st = np.tile(UNIFORM, 6)
    metrics = np.array([1.0, 0.0, 0.0, 1.0])
    out = np.zeros(5)
    assert po.oracle_lib().sfo_char_face_flux(6, dp(st), dp(metrics), po.WENO5, NEW_FLUXES[name], GAMMA,
                                              dp(out)) == 0
    assert all(near(out[v], PHYS_UNIFORM[v]) for v in range(5))


def test_rusanov_steger_lf_distinct_on_riemann_data(oracle):
    """Configured fluxes are observably distinct (test_numericalFlux.cpp:168-183)."""
    left = perfect_gas_state(1.0, 2.0, 0.1, 0.0, 1.0)
    right = perfect_gas_state(0.125, -0.5, 0.0, 0.0, 0.1)
    n = np.array([1.0, 0.0, 0.0])
    rus = np.zeros(5)
    po.oracle_lib().sfo_rusanov_flux(dp(left), dp(right), dp(n), GAMMA, dp(rus))
    sw, lf = _flux("Steger", left, right, n), _flux("LaxFriedrichs", left, right, n)
    for a, b in ((rus, sw), (rus, lf), (sw, lf)):
        assert not all(near(a[v], b[v], 1e-10) for v in range(5))


def test_lax_wendroff_needs_positive_dt_and_spacing(oracle):
    n = np.array([1.0, 0.0, 0.0])
    out = np.zeros(5)
    assert po.oracle_lib().sfo_lw_flux(dp(UNIFORM), dp(UNIFORM), dp(n), 0.0, 0.1, GAMMA, dp(out)) == po_err_arg()
    assert po.oracle_lib().sfo_lw_flux(dp(UNIFORM), dp(UNIFORM), dp(n), 1e-3, 0.0, GAMMA, dp(out)) == po_err_arg()


def po_err_arg():
    return [k for k, v in po.ERRORS.items() if v == "argument"][0]


@pytest.mark.skipif(not _ref_available(), reason="oracle/_ref not built (reference sources absent)")
def test_new_fluxes_bitwise_equal_reference(oracle):
    ref = po.ref_lib(False)
    rng = np.random.default_rng(0)
    for t in range(600):
        a = perfect_gas_state(*rng.uniform([0.1, -3, -3, -3, 0.1], [5, 3, 3, 3, 5]))
        b = perfect_gas_state(*rng.uniform([0.1, -3, -3, -3, 0.1], [5, 3, 3, 3, 5]))
        n = np.zeros(3)
        n[t % 3] = 1.0
        for name in NEW_FLUXES:
            want = np.zeros(5)
            if name == "Steger":
                ref.sfr_steger_flux(dp(a), dp(b), dp(n), GAMMA, dp(want))
            elif name == "LaxFriedrichs":
                ref.sfr_lf_flux(dp(a), dp(b), dp(n), GAMMA, dp(want))
            else:
                ref.sfr_lw_flux(dp(a), dp(b), dp(n), 1e-3, 0.1, GAMMA, dp(want))
            np.testing.assert_array_equal(_flux(name, a, b, n), want)


@pytest.mark.skipif(not _ref_available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("sname", ["weno3", "weno5", "teno5", "weno7"])
@pytest.mark.parametrize("fname", list(NEW_FLUXES))
def test_new_flux_operator_bitwise_equals_reference(oracle, sname, fname):
    """divDispatch with Steger-Warming / Lax-Friedrichs / Lax-Wendroff faces
    (the last with the step size set) against the restatement."""
    po.set_step_dt(2.5e-3)
    try:
        for gi, (dim, n, h) in enumerate(GRIDS):
            for bc in (po.BC_TRANSMISSIVE, po.BC_PERIODIC):
                q = smooth_state(dim, n, seed=200 + gi, shock=True)
                spec = po.GridSpec(dim=dim, n=n, ng=NG_OF[sname], h=h, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
                Q = spec.empty()
                spec.interior(Q)[...] = q
                po.fill_ghosts(spec, Q)
                rc = po.RefCase(spec, SCHEMES[sname], NEW_FLUXES[fname])
                np.testing.assert_array_equal(po.rhs(spec, SCHEMES[sname], NEW_FLUXES[fname], Q), rc.rhs(Q))
    finally:
        po.set_step_dt(0.0)


@pytest.mark.skipif(not _ref_available(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("fname", list(NEW_FLUXES))
def test_new_flux_time_loop_equals_reference(oracle, fname):
    spec = po.GridSpec(dim=1, n=(101, 1, 1), ng=3, h=(0.01, 1.0, 1.0))
    Q = spec.empty()
    x = np.arange(101) * 0.01
    I = spec.interior(Q)
    I[..., 0] = np.where(x < 0.5, 1.0, 0.125)
    I[..., 4] = np.where(x < 0.5, 1.0, 0.1) / 0.4
    Q2 = Q.copy()
    d1, t1 = po.advance(spec, po.WENO5, NEW_FLUXES[fname], po.SSPRK3, Q, 0.05, 0.4)
    d2, t2 = po.RefCase(spec, po.WENO5, NEW_FLUXES[fname]).advance(po.SSPRK3, Q2, 0.05, 0.4)
    np.testing.assert_array_equal(d1, d2)
    np.testing.assert_array_equal(Q, Q2)
