"""The host driver `sfg_run` on the GPU: a case directory in the reference's
format goes through the provider catalogs and the compiled plan to the
kernels, and the result matches the oracle run of the same case.

Tolerances: 1e-11 relative L-infinity per variable after a whole run (the
per-step bar of the parity tests is 1e-12; the run accumulates 875 steps);
plan mode (one C-ABI call per operation) and graph mode (sfg_advance) take
the same dt sequence, so their states agree to 1e-14.  The frozen-end golden
case is held to the bars its oracle meets (tests/test_oracle.py): integrals
2e-10, ranges 2e-7.
"""
import json
import os
import re
import subprocess

import numpy as np
import pytest

import pyoracle as po
from case_dirs import write_case
from conftest import rel_linf, rel_linf_vec

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "sonicsolver_b200", "sfg_run")
HERE = os.path.dirname(os.path.abspath(__file__))


def run_case(d, *args, dump=True):
    out = os.path.join(d, "final.bin")
    cmd = [RUNNER, d, *args] + (["--dump", out] if dump else [])
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    summary = json.loads(r.stdout.strip().splitlines()[-1])
    q = np.fromfile(out, dtype=np.float64) if dump else None
    return summary, q, r.stdout


def sod_oracle(cells=1000, t_end=0.2, cfl=0.5, write_interval=0.05):
    n = cells + 1
    h = 1.0 / cells
    spec = po.GridSpec(dim=1, n=(n, 1, 1), ng=3, h=(h, 0.1, 0.1), bc_lo=(0, 0, 0), bc_hi=(0, 0, 0))
    Q = spec.empty()
    I = spec.interior(Q)
    i = np.arange(n)
    I[0, 0, :, 0] = np.where(i < n // 2, 1.0, 0.125)
    I[0, 0, :, 4] = np.where(i < n // 2, 1.0, 0.1) / 0.4
    po.fill_ghosts(spec, Q)
    dts, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, t_end, cfl, write_interval=write_interval)
    return np.ascontiguousarray(spec.interior(Q)).reshape(-1, 5), dts, tf


@pytest.fixture(scope="module")
def sod_dir(tmp_path_factory):
    return write_case(str(tmp_path_factory.mktemp("cases")), "sod_c1", cells=(1000, 1, 1), box_hi=(1.0, 0.1, 0.1))


def test_sod_c1_case_directory_matches_oracle(sod_dir):
    s, q, out = run_case(sod_dir)
    want, dts, tf = sod_oracle()
    assert s["term_provider"] == "convection.conservativeFlux" and s["runtime_provider"] == "flow.conservative"
    assert s["steps"] == len(dts) and abs(s["time"] - tf) <= 1e-14 and s["status"] == 0
    assert rel_linf(q, want).max() <= 1e-11
    assert s["outputs"] == 4 and len(re.findall(r"^write t=", out, re.M)) == 4


def test_plan_mode_equals_graph_mode(sod_dir):
    g, qg, _ = run_case(sod_dir, "--mode", "graph", "--no-write")
    p, qp, _ = run_case(sod_dir, "--mode", "plan", "--no-write")
    assert g["steps"] == p["steps"] and g["time"] == p["time"]
    assert rel_linf(qp, qg).max() <= 1e-14


def _vts_arrays(text):
    """Name -> values of every DataArray of a .vts file (Points as "Points")."""
    out = {}
    pts = re.search(r"<Points>\s*<DataArray[^>]*>(.*?)</DataArray>", text, re.S)
    out["Points"] = np.array(pts.group(1).split(), dtype=np.float64)
    for m in re.finditer(r'<DataArray type="(\w+)" Name="([^"]+)"[^>]*>(.*?)</DataArray>', text, re.S):
        out[m.group(2)] = np.array(m.group(3).split(), dtype=np.int64 if m.group(1) == "Int32" else np.float64)
    return out


def test_vts_output_carries_the_state(sod_dir):
    """The output is the reference's result layout: the Field's nodes (the 1-D
    tube's unsolved y and z axes as their two node planes each), the
    boundary-set arrays, and Density / Pressure / Velocity (this case's
    registry declares no fields) with 17 digits."""
    s, q, _ = run_case(sod_dir)
    path = os.path.join(sod_dir, "result", "sod_c1_0003.vts")
    text = open(path).read()
    assert 'WholeExtent="0 1000 0 1 0 1"' in text and "TIME" not in text
    a = _vts_arrays(text)
    names = re.findall(r'Name="([^"]+)"', text)
    assert names == ["BC_ID", "BC_ID_rho", "BC_ID_U", "BC_ID_p", "Density", "Pressure", "Velocity"]
    q = q.reshape(-1, 5)
    rho = a["Density"].reshape(2, 2, 1001)
    for k in range(2):
        for j in range(2):
            np.testing.assert_array_equal(rho[k, j], q[:, 0])   # 17 digits round-trip exactly
    np.testing.assert_array_equal(a["Velocity"].reshape(2, 2, 1001, 3)[0, 0, :, 0], q[:, 1] / q[:, 0])
    pts = a["Points"].reshape(2, 2, 1001, 3)
    assert pts[1, 1, 1000].tolist() == [1.0, 0.1, 0.1] and pts[0, 0, 0].tolist() == [0.0, 0.0, 0.0]
    # Left = 1, Right = 2, sideWalls = 3, frontBack = 4: the empty patches'
    # node planes cover every node of the tube, the last-named set wins
    assert (a["BC_ID"] == 4).all() and (a["BC_ID_rho"] == 4).all()
    assert "1=Left, 2=Right, 3=sideWalls, 4=frontBack;" in text


def test_vts_boundary_sets_and_declared_fields(tmp_path):
    """A 2-D box whose registry declares U and rho for output and p not:
    U and rho take those names, Pressure keeps its built-in name; boundary
    sets are numbered by first appearance over the rho, U, p conditions and
    a later condition wins on shared nodes."""
    bnd = {"frontBack": "empty", "Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "zeroGradient"}
    d = write_case(str(tmp_path), "sets", cells=(30, 10, 1), box_hi=(3.0, 1.0, 0.1), end_time=0.01,
                   write_interval=0.01, boundaries=bnd)
    with open(os.path.join(d, "fields", "fields.yaml"), "a") as f:
        f.write("U:\n  type: vector\n  output: true\nrho:\n  type: scalar\n  output: true\n"
                "p:\n  type: scalar\n  output: false\n")
    s, q, _ = run_case(d)
    vts = sorted(f for f in os.listdir(os.path.join(d, "result")) if f.endswith(".vts"))
    text = open(os.path.join(d, "result", vts[-1])).read()
    names = re.findall(r'Name="([^"]+)"', text)
    assert names[4:] == ["Pressure", "U", "rho"]
    a = _vts_arrays(text)
    # frontBack = 1 (both node planes of the one-cell-deep box: every node),
    # Left = 2, Right = 3, sideWalls = 4
    assert "1=frontBack, 2=Left, 3=Right, 4=sideWalls;" in text
    ids = a["BC_ID"].reshape(2, 11, 31)
    assert ids[0, 5, 0] == 2 and ids[1, 5, 30] == 3 and ids[0, 10, 5] == 4 and ids[1, 5, 5] == 1
    assert ids[0, 0, 0] == 4 and ids[1, 10, 30] == 4   # corners: sideWalls, the last condition, wins
    np.testing.assert_array_equal(a["rho"].reshape(2, 11, 31)[1].ravel(), q.reshape(-1, 5)[:, 0])


# ------------------------------------------------- frozen end (no condition)

def _weighted_integrals(q, nx, ny, gamma):
    """Trapezoid node integrals of the reference's output check (2 z-nodes of
    weight 0.5 at dz = 0.1), as tests/test_oracle.py computes them."""
    I = q.reshape(ny, nx, 5)
    rho = I[..., 0]
    u, v, w = I[..., 1] / rho, I[..., 2] / rho, I[..., 3] / rho
    p = (gamma - 1.0) * (I[..., 4] - 0.5 * rho * (u * u + v * v + w * w))
    W = np.ones(rho.shape)
    W[:, 0] *= 0.5
    W[:, -1] *= 0.5
    W[0, :] *= 0.5
    W[-1, :] *= 0.5
    W *= 0.5 * 0.1 * 2
    sp = np.sqrt(u * u + v * v + w * w)
    return {"rho": (rho.min(), rho.max()), "p": (p.min(), p.max()), "speed": (sp.min(), sp.max()),
            "mass": (W * rho).sum(), "momentum": [(W * I[..., k]).sum() for k in (1, 2, 3)],
            "energy": (W * I[..., 4]).sum()}


def test_reference_sod_golden_case_through_the_plan(tmp_path):
    """The reference's frozen-ghost WENO7 + Rusanov + forwardEuler Sod case
    (100 x 20 cells, no Left condition), written as a case directory from the
    committed fixture and run by sfg_run: 454 steps, t = 0.2, the baseline's
    integrals and ranges, and the oracle's final state."""
    with open(os.path.join(HERE, "golden", "sod_weno7_t0p2.json")) as f:
        fx = json.load(f)
    c, base = fx["case"], fx["baseline"]
    L = c["left"], c["right"]
    d = write_case(str(tmp_path), "sod_weno7", cells=tuple(c["cells"]), box_hi=tuple(c["length"]),
                   n_ghost=c["n_ghost"], convection=c["recipe"], time=c["time"], end_time=c["t_end"], cfl=c["cfl"],
                   write_interval=c["write_interval"], gamma=c["gamma"],
                   left=(L[0]["rho"], L[0]["u"], L[0]["p"]), right=(L[1]["rho"], L[1]["u"], L[1]["p"]),
                   boundaries={"Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"})
    s, q, out = run_case(d, "--no-write")
    nx, ny, _ = c["nodes"]
    assert "bc=20/00/00" in out and s["nodes"] == [nx, ny, 1]
    assert s["steps"] == base["steps"] == 454 and abs(s["time"] - base["final_time"]) <= 5e-12
    got = _weighted_integrals(q, nx, ny, c["gamma"])
    for k in ("rho", "p", "speed"):
        for a, b in zip(got[k], base["ranges"][k]):
            assert abs(a - b) <= 2e-7 * abs(b), (k, a, b)
    for k in ("mass", "energy"):
        assert abs(got[k] - base["integrals"][k]) <= 2e-10 * base["integrals"][k], k
    mx = base["integrals"]["momentum"][0]
    assert abs(got["momentum"][0] - mx) <= 2e-10 * mx
    assert abs(got["momentum"][1]) < 1e-7 and got["momentum"][2] == 0.0
    from test_oracle import _sod_run
    _, spec, Q, dts, tf = _sod_run()
    want = np.ascontiguousarray(spec.interior(Q)).reshape(-1, 5)
    assert len(dts) == s["steps"]
    assert rel_linf(q, want).max() <= 1e-9


def _frozen_pair(recipe="weno5Rusanov", n=(40, 12, 1), h=(0.02, 0.03, 1.0), ghost_state=None, seed=4):
    from helpers import FLUX_OF, SCHEME_OF, smooth_state, split_recipe
    from sonicsolver_b200 import capi
    scheme, flux = split_recipe(recipe)
    ng = 4 if scheme == "weno7" else 3
    lo, hi = (po.BC_FROZEN, po.BC_TRANSMISSIVE, 0), (po.BC_TRANSMISSIVE, po.BC_TRANSMISSIVE, 0)
    spec = po.GridSpec(dim=2, n=n, ng=ng, h=h, bc_lo=lo, bc_hi=hi)
    q = smooth_state(2, n, seed=seed, shock=True)
    Q = spec.empty()                   # oracle Field: (1, ny + 2 ng, nx + 2 ng, 5)
    spec.interior(Q)[...] = q.reshape(spec.interior(Q).shape)
    Q[:, :, :ng] = Q[:, :, ng:ng + 1] if ghost_state is None else ghost_state   # frozen x-low ghosts
    po.fill_ghosts(spec, Q)
    s = capi.Solver(2, n, h, (capi.BC_FROZEN, capi.BC_TRANSMISSIVE, 0), (capi.BC_TRANSMISSIVE,) * 2 + (0,),
                    recipe=recipe, time_recipe="SSPRK3")
    if ghost_state is None:
        s.upload(np.ascontiguousarray(q))
    else:                              # C-ABI Field layout: ng ghosts on every axis, z included
        F = np.zeros((1 + 2 * ng,) + Q.shape[1:])
        F[ng] = Q[0]
        s.upload(np.ascontiguousarray(F), layout=capi.LAYOUT_FIELD)
    return spec, Q, s, po.Stepper(spec, SCHEME_OF[scheme], FLUX_OF[flux], po.SSPRK3), q.shape


@pytest.mark.parametrize("recipe", ["weno5Rusanov", "teno5Roe", "weno7Rusanov"])
def test_frozen_end_steps_match_oracle(recipe):
    spec, Q, s, st, shape = _frozen_pair(recipe)
    for _ in range(5):
        dt = po.dt(spec, Q, 0.5)
        assert abs(s.compute_dt() - dt) <= 1e-14 * dt
        st.step(Q, dt)
        s.step(dt)
    got = s.download().reshape(-1, 5)
    assert got.shape[0] == 40 * 12     # the device's extra node is not part of the caller's grid
    assert rel_linf(got, np.ascontiguousarray(spec.interior(Q)).reshape(-1, 5)).max() <= 1e-12


def test_frozen_end_field_layout_ghosts_are_used():
    """Field-layout upload: the frozen ghosts keep the values the caller
    gave (here a different state from the boundary node), as the reference
    does; download writes them back unchanged."""
    from sonicsolver_b200 import capi
    ghost = np.array([1.3, 0.2, 0.0, 0.0, 2.9])
    spec, Q, s, st, shape = _frozen_pair(ghost_state=ghost)
    dt = po.dt(spec, Q, 0.5)
    assert abs(s.compute_dt() - dt) <= 1e-14 * dt
    st.step(Q, dt)
    s.step(dt)
    ng = spec.ng
    got = s.download(layout=capi.LAYOUT_FIELD).reshape((1 + 2 * ng,) + Q.shape[1:])[ng]
    assert rel_linf(got[ng:-ng, ng:-ng], spec.interior(Q)[0]).max() <= 1e-12
    np.testing.assert_array_equal(got[ng:-ng, :ng], np.broadcast_to(ghost, got[ng:-ng, :ng].shape))


LAW_CASE = {
    "Left": {"rho": "fixedValue: 1.0", "U": "fixedValue: [0.3 0 0]", "p": "fixedValue: 1.0"},
    "Right": {"rho": "zeroGradient", "U": "noSlip", "p": "zeroGradient"},
    "sideWalls": "empty", "frontBack": "empty",
}


def law_oracle(cells=400, t_end=0.1, cfl=0.5, write_interval=0.05):
    """The law case of LAW_CASE on the oracle: inflow on the left, a wall on
    the right; ghosts start as copies of the boundary nodes, as the device's
    upload holds them."""
    n = cells + 1
    h = 1.0 / cells
    laws = {(0, 0): po.LawSpec(po.LAW_FIXED_VALUE, po.LAW_FIXED_VALUE, po.LAW_FIXED_VALUE, rho_value=1.0,
                               U_value=(0.3, 0.0, 0.0), p_value=1.0),
            (0, 1): po.LawSpec(po.LAW_ZERO_GRADIENT, po.LAW_FIXED_VALUE, po.LAW_ZERO_GRADIENT)}
    spec = po.GridSpec(dim=1, n=(n, 1, 1), ng=3, h=(h, 0.1, 0.1), bc_lo=(po.BC_LAW, 0, 0),
                       bc_hi=(po.BC_LAW, 0, 0), laws=laws)
    Q = spec.empty()
    i = np.arange(n)
    Q[0, 0, 3:3 + n, 0] = np.where(i < n // 2, 1.0, 0.125)
    Q[0, 0, 3:3 + n, 4] = np.where(i < n // 2, 1.0, 0.1) / 0.4
    Q[0, 0, :3] = Q[0, 0, 3]
    Q[0, 0, 3 + n:] = Q[0, 0, 2 + n]
    dts, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, t_end, cfl, write_interval=write_interval)
    return np.ascontiguousarray(spec.interior(Q)).reshape(-1, 5), dts, tf


@pytest.fixture(scope="module")
def law_dir(tmp_path_factory):
    return write_case(str(tmp_path_factory.mktemp("cases")), "law_c1", cells=(400, 1, 1), box_hi=(1.0, 0.1, 0.1),
                      end_time=0.1, write_interval=0.05, boundaries=LAW_CASE)


@pytest.mark.parametrize("mode", ["graph", "plan"])
def test_law_case_directory_matches_oracle(law_dir, mode):
    """fixedValue inflow and a noSlip wall from case.yaml through sfg_run:
    the laws run before every step and stage and after each step, as the
    reference's FlowStepPrepare / stage RHS / FlowStepCommit apply them."""
    s, q, _ = run_case(law_dir, "--mode", mode, "--no-write")
    want, dts, tf = law_oracle()
    assert s["steps"] == len(dts) and abs(s["time"] - tf) <= 1e-14 and s["status"] == 0
    assert rel_linf(q, want).max() <= 1e-11
    q = q.reshape(-1, 5)
    assert q[0, 0] == 1.0 and q[0, 1] == 0.3 and q[-1, 1] == 0.0


# ---- graded and curved blocks through the case reader

TWO_D = {"Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"}
CURVED_BLOCKS = {
    # a graded box (trilinear interpolation; the grading is the ratio of
    # neighbouring cell sizes)
    "graded": dict(cells=(48, 32, 1), box_hi=(1.2, 0.8, 0.1), grading=(1.02, 0.985, 1.0)),
    # a skewed quadrilateral prism
    "skewed": dict(cells=(40, 30, 1), box_hi=(1, 1, 1),
                   vertices=[[0.0, 0.0, 0.0], [1.2, 0.15, 0.0], [1.35, 0.95, 0.0], [-0.1, 0.8, 0.0],
                             [0.0, 0.0, 0.1], [1.2, 0.15, 0.1], [1.35, 0.95, 0.1], [-0.1, 0.8, 0.1]]),
    # an annular sector with arc edges (transfinite interpolation), the shape
    # of the reference's createMesh blocks, one cell deep
    "arc": dict(cells=(40, 20, 1), box_hi=(1, 1, 1),
                vertices=[[0.67175144, 0.67175144, 0.0], [-0.67175144, 0.67175144, 0.0], [-0.4, 0.4, 0.0],
                          [0.4, 0.4, 0.0], [0.67175144, 0.67175144, 0.01], [-0.67175144, 0.67175144, 0.01],
                          [-0.4, 0.4, 0.01], [0.4, 0.4, 0.01]],
                edges=[(0, 1, (0.0, 0.95, 0.0)), (4, 5, (0.0, 0.95, 0.01))]),
}
CURVED_T_END, CURVED_WRITE, CURVED_CFL = 0.06, 0.03, 0.45


def curved_oracle(kw, metrics_file):
    """The Sod problem of a curved-block case on the oracle, with the
    metrics sfg_run handed to the provider (the node plane of the inactive
    axis)."""
    nx, ny = kw["cells"][0] + 1, kw["cells"][1] + 1
    ng = 3
    M = np.fromfile(metrics_file).reshape(1 + 2 * ng, ny + 2 * ng, nx + 2 * ng, 10)[ng:ng + 1]
    spec = po.GridSpec(dim=2, n=(nx, ny, 1), ng=ng, h=(1.0, 1.0, 1.0), metrics=M)
    Q = spec.empty()
    I = spec.interior(Q)
    left = np.arange(nx) < nx // 2
    I[..., 0] = np.where(left, 1.0, 0.125)
    I[..., 4] = np.where(left, 1.0, 0.1) / 0.4
    po.fill_ghosts(spec, Q)
    dts, tf = po.advance(spec, po.WENO5, po.RUSANOV, po.SSPRK3, Q, CURVED_T_END, CURVED_CFL,
                         write_interval=CURVED_WRITE)
    return np.ascontiguousarray(spec.interior(Q)).reshape(-1, 5), dts, tf


@pytest.mark.parametrize("block", sorted(CURVED_BLOCKS))
@pytest.mark.parametrize("mode", ["graph", "plan"])
def test_curved_block_case_directory_matches_oracle(tmp_path, block, mode):
    """A graded, a skewed and an arc-edged 2-D block read from case.yaml:
    sfg_run builds the generator's node coordinates and conservative
    metrics, hands them to the provider in the Field layout, and runs a Sod
    problem along the block's first axis; the oracle runs the same problem
    on the metrics sfg_run dumps, with the same output times."""
    kw = CURVED_BLOCKS[block]
    d = write_case(str(tmp_path), block, end_time=CURVED_T_END, write_interval=CURVED_WRITE, cfl=CURVED_CFL,
                   boundaries=TWO_D, **kw)
    fm = os.path.join(d, "metrics.bin")
    s, q, out = run_case(d, "--mode", mode, "--no-write", "--dump-metrics", fm)
    assert "mesh curvilinear" in out and s["status"] == 0
    want, dts, tf = curved_oracle(kw, fm)
    assert s["steps"] == len(dts) and abs(s["time"] - tf) <= 1e-14
    # momentum against one scale: rho v of the graded box stays at round-off
    assert rel_linf_vec(q, want).max() <= 1e-11


def test_curved_block_vts_carries_the_generated_points(tmp_path):
    """The .vts output of a curved block holds the generated node
    coordinates, not a box."""
    kw = CURVED_BLOCKS["arc"]
    d = write_case(str(tmp_path), "arcvts", end_time=0.01, write_interval=0.01, boundaries=TWO_D, **kw)
    fp = os.path.join(d, "points.bin")
    run_case(d, "--dump-points", fp, dump=False)
    vts = sorted(f for f in os.listdir(os.path.join(d, "result")) if f.endswith(".vts"))
    with open(os.path.join(d, "result", vts[-1])) as f:
        text = f.read()
    pts = _vts_arrays(text)["Points"].reshape(2, 21, 41, 3)   # both node planes of the one-cell-deep block
    assert np.array_equal(pts[0].ravel(), np.fromfile(fp))
    # the second plane: z = 0.01, the same x, y (to the round-off of the
    # transfinite sums)
    assert np.abs(pts[1, ..., 2] - 0.01).max() <= 1e-15 and np.abs(pts[1, ..., :2] - pts[0, ..., :2]).max() <= 1e-14


# ---- several case directories on the batched provider

def test_batch_mode_equals_single_case_runs(tmp_path):
    """`sfg_run --batch` over case directories of every end kind (a law
    tube, a tube without a Left condition, a 2-D box on TENO5 + Roe with its
    own CFL, and a forwardEuler WENO7 case in a second batch): each ends at
    its own endTime with the step count and the time of its single-case run
    (output clipping included) and its final state within 1e-12 (the same
    bits on the tile kernels; a 1-D FP64 case alone may take the whole-run
    cluster kernel, equal to round-off)."""
    root = str(tmp_path)
    box = {"Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"}
    frozen = {"Right": "zeroGradient", "sideWalls": "empty", "frontBack": "empty"}
    dirs = [write_case(root, "law", cells=(400, 1, 1), box_hi=(1.0, 0.1, 0.1), end_time=0.1, write_interval=0.05,
                       boundaries=LAW_CASE),
            write_case(root, "frozen", cells=(300, 1, 1), box_hi=(1.0, 0.1, 0.1), end_time=0.08, write_interval=0.03,
                       boundaries=frozen),
            write_case(root, "box", cells=(48, 24, 1), box_hi=(2.0, 1.0, 0.1), end_time=0.07, write_interval=0.02,
                       cfl=0.4, convection="teno5Roe", boundaries=box),
            write_case(root, "euler7", cells=(100, 20, 1), box_hi=(100.0, 20.0, 0.1), n_ghost=4, end_time=0.05,
                       write_interval=0.05, convection="weno7Rusanov", time="forwardEuler",
                       left=(1.0, 0.0, 1e5), right=(0.125, 0.0, 1e4),
                       boundaries={"Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"})]
    dump = os.path.join(root, "dump")
    os.makedirs(dump)
    r = subprocess.run([RUNNER, "--batch", *dirs, "--dump-dir", dump, "--no-write"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert [l["case"] for l in lines] == ["law", "frozen", "box", "euler7"]
    assert "batch time=SSPRK3 cases=3" in r.stdout and "batch time=forwardEuler cases=1" in r.stdout
    for d, got in zip(dirs, lines):
        alone, q, _ = run_case(d, "--no-write")
        assert got["status"] == 0 and got["steps"] == alone["steps"], (got, alone)
        assert abs(got["time"] - alone["time"]) <= 1e-14
        qb = np.fromfile(os.path.join(dump, got["case"] + ".bin"))
        assert rel_linf_vec(qb, q).max() <= 1e-12, got["case"]
