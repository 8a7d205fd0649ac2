"""The C++17 host side (case reader, provider catalogs, plan, driver) on the
CPU: `sfg_run --selftest` checks the catalog and plan rules, `--describe`
reads a case directory, resolves its providers and validates the plan
bindings without touching a GPU."""
import os
import subprocess

import numpy as np

import pytest

from case_dirs import write_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "sonicsolver_b200", "sfg_run")
# the reference's own case directories, read in place when present
# (SONICSOLVER_REFERENCE overrides the tree's location)
REFERENCE_TESTS = os.path.join(os.environ.get("SONICSOLVER_REFERENCE", "/root/reference"), "test")


@pytest.fixture(scope="module")
def runner():
    from sonicsolver_b200 import build
    build.build_host()
    return RUNNER


def run(runner, *args):
    return subprocess.run([runner, *args], capture_output=True, text=True, timeout=60)


def test_selftest(runner):
    r = run(runner, "--selftest")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "selftest passed" in r.stdout and "FAILED" not in r.stdout


@pytest.mark.parametrize("form", ["terms", "scheme"])
def test_describe_sod_case(runner, tmp_path, form):
    d = write_case(str(tmp_path), "sod", cells=(1000, 1, 1), box_hi=(1.0, 0.1, 0.1), numerics_form=form)
    r = run(runner, d, "--describe")
    assert r.returncode == 0, r.stderr
    assert "convection.conservativeFlux" in r.stdout and "recipe weno5Rusanov" in r.stdout
    assert "grid dim=1 nodes=1001,1,1 h=0.001," in r.stdout and "bc=00/00/00" in r.stdout
    for op in ("flow.step.prepare", "flow.dt.compute", "flow.step.begin", "explicit.stage.execute",
               "flow.step.commit", "time.commit"):
        assert f"[{op} @ flow.conservative]" in r.stdout
    assert "stage-loop Explicit.stages x3" in r.stdout and "bindings valid" in r.stdout


def test_describe_2d_frozen_and_periodic(runner, tmp_path):
    d = write_case(str(tmp_path), "frozen", cells=(100, 20, 1), box_hi=(100.0, 20.0, 0.1), n_ghost=4,
                   convection="weno7Rusanov", time="forwardEuler",
                   boundaries={"Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"})
    r = run(runner, d, "--describe")
    assert r.returncode == 0, r.stderr
    assert "grid dim=2 nodes=101,21,1 h=1,1," in r.stdout and "bc=20/00/00" in r.stdout   # Left: frozen
    d2 = write_case(str(tmp_path), "periodic", cells=(64, 32, 1), box_hi=(1.0, 0.5, 0.1),
                    boundaries={"Left": "periodic", "Right": "periodic", "sideWalls": "periodic",
                                "frontBack": "empty"})
    r2 = run(runner, d2, "--describe")
    assert r2.returncode == 0 and "nodes=64,32,1" in r2.stdout and "bc=11/11/00" in r2.stdout


@pytest.mark.parametrize("convection,needle", [("weno5Roeish", "no term provider"),
                                               ("upwind1Rusanov", "no term provider")])
def test_unsupported_recipe(runner, tmp_path, convection, needle):
    d = write_case(str(tmp_path), "c", cells=(50, 1, 1), box_hi=(1.0, 0.1, 0.1), convection=convection)
    r = run(runner, d, "--describe")
    assert r.returncode == 3 and needle in r.stderr


def test_unsupported_condition_and_time(runner, tmp_path):
    d = write_case(str(tmp_path), "a", cells=(50, 1, 1), box_hi=(1.0, 0.1, 0.1),
                   boundaries={"Left": "inletOutlet", "Right": "zeroGradient", "sideWalls": "empty",
                               "frontBack": "empty"})
    r = run(runner, d, "--describe")
    assert r.returncode == 3 and "inletOutlet" in r.stderr
    d2 = write_case(str(tmp_path), "b", cells=(50, 1, 1), box_hi=(1.0, 0.1, 0.1), time="backwardEuler")
    r2 = run(runner, d2, "--describe")
    assert r2.returncode == 3 and "time recipe" in r2.stderr


def test_parse_error_names_file_and_line(runner, tmp_path):
    d = write_case(str(tmp_path), "bad", cells=(50, 1, 1), box_hi=(1.0, 0.1, 0.1))
    with open(os.path.join(d, "solvers", "runtime.yaml"), "a") as f:
        f.write("this line has no colon\n")
    r = run(runner, d, "--describe")
    assert r.returncode == 1 and "runtime.yaml:" in r.stderr


@pytest.mark.skipif(not os.path.isdir(REFERENCE_TESTS), reason="reference case directories not present")
def test_reference_case_directories(runner):
    """Every case directory of the reference's test tree is read without a
    parse error.  The three Sod cases (no Left condition: frozen ghosts;
    TENO5 + Steger-Warming and WENO7 + Rusanov) and the inviscid GUI Sod case
    resolve and plan; every other case is reported as not supported by this
    provider, with its reason (the immersed-boundary, thermal and mixture
    cases by the physics they switch on, although their meshes would run)."""
    dirs = sorted(os.path.dirname(os.path.join(dp, f)) for dp, _, fs in os.walk(REFERENCE_TESTS)
                  for f in fs if f == "case.yaml")
    assert len(dirs) > 10
    resolved = []
    for d in dirs:
        r = run(runner, d, "--describe")
        rel = os.path.relpath(d, REFERENCE_TESTS)
        assert r.returncode in (0, 3), (rel, r.returncode, r.stderr)
        if r.returncode == 0:
            assert "bindings valid" in r.stdout
            resolved.append(rel)
            if rel.startswith("Sod" + os.sep):
                assert "bc=20/00/00" in r.stdout
        else:
            assert "unsupported:" in r.stderr
    assert sorted(resolved) == sorted([os.path.join("Sod", c) for c in
                                       ("sodCase", "sodCase_weno7", "sodCase_weno7_t0p2")] +
                                      [os.path.join("guiCase", "sodGuiFromSfm")])
    reasons = {"thermalCase": "temperature equation", "mixtureCase": "multiphase flow",
               "variationalIBMCase": "immersed boundary",
               os.path.join("IBM", "cylinderFlowPeskin"): "viscous terms"}
    for rel, why in reasons.items():
        r = run(runner, os.path.join(REFERENCE_TESTS, rel), "--describe")
        assert r.returncode == 3 and why in r.stderr, (rel, r.stderr)


def _add_module(d, name, body):
    """Registers models/<name>.yaml (type <name>) with `body` in a case."""
    with open(os.path.join(d, "models", "models.yaml"), "a") as f:
        f.write(f"{name}:\n  type: {name}\n  file: models/{name}.yaml\n")
    with open(os.path.join(d, "models", f"{name}.yaml"), "w") as f:
        f.write(f"SonicFile:\n  object: models\n  type: {name}\n" + body)


@pytest.mark.parametrize("module,body,why", [
    ("IBM", "IBM:\n  enabled: true\n  type: ghost\n", "immersed boundary"),
    ("turbulence", "enabled: true\nsimulationType: RAS\n", "turbulence model (simulationType 'RAS')"),
    ("multiPhase", "multiPhases: true\n", "multiphase flow"),
    ("phaseChange", "phaseChange:\n  enabled: true\n", "phase change"),
    ("thermophysical", "temperature:\n  enabled: true\n  fieldName: T\n", "temperature equation"),
])
def test_physics_gate_refuses_enabled_modules(runner, tmp_path, module, body, why):
    """A model module that switches on physics beyond the inviscid Euler
    equations makes the case unsupported (exit 3, the reason on stderr)."""
    d = write_case(str(tmp_path), "gate", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1))
    assert run(runner, d, "--describe").returncode == 0
    _add_module(d, module, body)
    r = run(runner, d, "--describe")
    assert r.returncode == 3 and why in r.stderr, r.stderr


def test_physics_gate_inert_modules(runner, tmp_path):
    """Disabled modules, a laminar or DNS turbulence entry, gravity (which
    acts only through numerics sources) and a diffusion scheme switched off
    by transport.enable: false leave the case runnable; a live diffusion
    scheme or a numerics source term does not."""
    d = write_case(str(tmp_path), "inert", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1), numerics_form="scheme")
    _add_module(d, "IBM", "IBM:\n  enabled: false\n")
    _add_module(d, "turbulence", "enabled: true\nsimulationType: DNS\n")
    _add_module(d, "gravity", "value: [9.8, 0, 0]\n")
    _add_module(d, "thermophysical", "temperature:\n  enabled: false\n")
    r = run(runner, d, "--describe")
    assert r.returncode == 0, r.stderr
    num = os.path.join(d, "solvers", "numerics.yaml")
    text = open(num).read()
    with open(num, "w") as f:
        f.write(text.replace("  enable: false\n", ""))
    r = run(runner, d, "--describe")
    assert r.returncode == 3 and "viscous terms" in r.stderr, r.stderr
    with open(num, "w") as f:
        f.write(text + "sources:\n  default: Gravity\n")
    r = run(runner, d, "--describe")
    assert r.returncode == 3 and "source terms 'Gravity'" in r.stderr, r.stderr


LAW_BOUNDARIES = {
    "Left": {"rho": "fixedValue: 1.2", "U": "fixedValue: [0.5 0 0]", "p": "fixedValue: 1.1"},
    "Right": {"rho": "zeroGradient", "U": "noSlip", "p": "{type: zeroGradient}"},
    "sideWalls": "empty", "frontBack": "empty",
}


def test_describe_law_patches(runner, tmp_path):
    """fixedValue / noSlip / zeroGradient per field become SFG_BC_LAW ends
    with those laws; the compact SonicFile syntax is read."""
    d = write_case(str(tmp_path), "laws", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1), boundaries=LAW_BOUNDARIES)
    r = run(runner, d, "--describe")
    assert r.returncode == 0, r.stderr
    assert "bc=33/00/00" in r.stdout
    assert "law xlo rho=fixedValue(1.2) U=fixedValue(0.5,0,0) p=fixedValue(1.1000000000000001)" in r.stdout
    assert "law xhi rho=zeroGradient(0) U=fixedValue(0,0,0) p=zeroGradient(0)" in r.stdout
    slip = dict(LAW_BOUNDARIES, Right={"rho": "zeroGradient", "U": "slip", "p": "symmetry"})
    r2 = run(runner, write_case(str(tmp_path), "slip", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1), boundaries=slip),
             "--describe")
    assert r2.returncode == 0 and "law xhi rho=zeroGradient(0) U=symmetry(0,0,0) p=symmetry(0)" in r2.stdout
    # all-zeroGradient patches stay transmissive
    zg = dict(LAW_BOUNDARIES, Left={"rho": "zeroGradient", "U": "zero_gradient", "p": "ZeroGradient"})
    r3 = run(runner, write_case(str(tmp_path), "zg", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1), boundaries=zg),
             "--describe")
    assert r3.returncode == 0 and "bc=03/00/00" in r3.stdout


def test_law_patch_errors(runner, tmp_path):
    partial = dict(LAW_BOUNDARIES, Right={"U": "noSlip"})
    r = run(runner, write_case(str(tmp_path), "partial", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1),
                               boundaries=partial), "--describe")
    assert r.returncode == 3 and "rho has no condition" in r.stderr
    bad = dict(LAW_BOUNDARIES, Left={"rho": "fixedValue: 1.2", "U": "fixedValue: 0.5", "p": "fixedValue: 1.1"})
    r2 = run(runner, write_case(str(tmp_path), "bad", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1), boundaries=bad),
             "--describe")
    assert r2.returncode == 1 and "fixedValue needs 3 number(s)" in r2.stderr
    noslip_p = dict(LAW_BOUNDARIES, Right={"rho": "zeroGradient", "U": "noSlip", "p": "noSlip"})
    r3 = run(runner, write_case(str(tmp_path), "np", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1),
                                boundaries=noslip_p), "--describe")
    assert r3.returncode == 3 and "noSlip" in r3.stderr


# ---- graded and curved blocks: the generator's node coordinates and metrics

CREATEMESH = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "createmesh_blocks.npz"))
ALL_ZG = {"Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "zeroGradient"}
TWO_D = {"Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "zeroGradient", "frontBack": "empty"}


def _dump(runner, d, *flags):
    r = run(runner, d, "--describe", *flags)
    assert r.returncode == 0, r.stdout + r.stderr
    return r.stdout


def _sixth_digit(want):
    """One unit in the sixth significant digit of each value (the
    reference's .vts files print coordinates with six digits)."""
    a = np.abs(want)
    return np.where(a > 0, 10.0 ** (np.floor(np.log10(np.where(a > 0, a, 1.0))) - 5), 0.0) + 1e-12


@pytest.mark.parametrize("block", [0, 1, 2])
def test_createmesh_blocks_match_the_reference_generator(runner, tmp_path, block):
    """Blocks 0-2 of the reference's createMesh case (a box whose hex runs
    against the axes; two 40 x 20 x 190 hexes with arc edges, transfinite
    interpolation): the node coordinates equal the reference generator's
    own .vts output to its six printed digits."""
    g = CREATEMESH
    edges = [(int(a), int(b), p) for (a, b), p in zip(g["edge_vertices"], g["edge_points"])]
    c = g[f"cells_{block}"]
    d = write_case(str(tmp_path), f"blk{block}", cells=tuple(int(x) for x in c), box_hi=(1, 1, 1),
                   vertices=g["vertices"], hex=g[f"hex_{block}"], grading=g[f"grading_{block}"], edges=edges,
                   boundaries=ALL_ZG)
    f = os.path.join(str(tmp_path), "points.bin")
    out = _dump(runner, d, "--dump-points", f)
    assert "mesh curvilinear (transfinite, arc edges)" in out
    P = np.fromfile(f).reshape(c[2] + 1, c[1] + 1, c[0] + 1, 3)[g["planes"]]
    want = g[f"points_{block}"]
    assert (np.abs(P - want) <= _sixth_digit(want)).all()
    # the printed digits themselves agree almost everywhere (the rest sit on
    # a rounding boundary or are round-off around zero)
    printed = np.array([float("%g" % v) for v in P.ravel()]).reshape(P.shape)
    assert (printed == want).mean() > 0.98


def test_graded_block_points_and_metrics(runner, tmp_path):
    """A graded box (no edges: trilinear interpolation with the generator's
    geometric grading): node coordinates follow x_i = x0 + L (1 - g^i) /
    (1 - g^n), and the symmetric conservative metrics of the orthogonal
    grid are xi_x = 2 / (x_i+1 - x_i-1) (likewise eta_y, zeta_z), zero
    cross terms, Jac = 1 / J the product of the central spacings; the
    metric identity audit passes."""
    cells, grading, lo, hi = (12, 8, 6), (2.0, 0.5, 1.3), (-0.5, 0.25, 1.0), (1.5, 1.0, 1.6)
    d = write_case(str(tmp_path), "graded", cells=cells, box_lo=lo, box_hi=hi, grading=grading, boundaries=ALL_ZG)
    fp, fm = os.path.join(str(tmp_path), "p.bin"), os.path.join(str(tmp_path), "m.bin")
    out = _dump(runner, d, "--dump-points", fp, "--dump-metrics", fm)
    assert "mesh curvilinear (trilinear, graded)" in out
    nodes = [c + 1 for c in cells]
    P = np.fromfile(fp).reshape(nodes[2], nodes[1], nodes[0], 3)
    axes = []
    for a in range(3):
        t = (1 - grading[a] ** np.arange(nodes[a])) / (1 - grading[a] ** cells[a])
        axes.append(lo[a] + (hi[a] - lo[a]) * t)
    Z, Y, X = np.meshgrid(axes[2], axes[1], axes[0], indexing="ij")
    for a, want in enumerate((X, Y, Z)):
        assert np.abs(P[..., a] - want).max() <= 4e-14
    e = [n + 6 for n in nodes]
    M = np.fromfile(fm).reshape(e[2], e[1], e[0], 10)[3:-3, 3:-3, 3:-3]     # the nodes
    dc = [(ax[2:] - ax[:-2]) / 2 for ax in axes]                            # central spacings of inner nodes
    DZ, DY, DX = np.meshgrid(dc[2], dc[1], dc[0], indexing="ij")
    Mi = M[1:-1, 1:-1, 1:-1]
    for comp, dd in ((1, DX), (5, DY), (9, DZ)):
        assert np.abs(Mi[..., comp] * dd - 1).max() <= 1e-13
    for comp in (2, 3, 4, 6, 7, 8):
        assert np.abs(Mi[..., comp]).max() <= 1e-12 * np.abs(Mi[..., (1, 5, 9)]).max()
    assert np.abs(Mi[..., 0] * DX * DY * DZ - 1).max() <= 1e-13
    line = out.split("metric identity residual ")[1].splitlines()[0]
    res, tol = [float(v) for v in line.split(", tolerance ")]
    assert res <= tol


def test_block_orientation_and_curved_limits(runner, tmp_path):
    """A box listed in the canonical corner order runs on the uniform path;
    the same box with its hex listed against the axes takes the generated
    coordinates; periodic ends on a curved block are refused (the reference
    has no periodic boundary there)."""
    out = _dump(runner, write_case(str(tmp_path), "box", cells=(16, 8, 1), box_hi=(2.0, 1.0, 0.1),
                                   boundaries=TWO_D))
    assert "mesh curvilinear" not in out and "dim=2 nodes=17,9,1 h=0.125,0.125," in out
    verts = [[2.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 1.0, 0.0], [2.0, 1.0, 0.0],
             [2.0, 0.0, 0.1], [0.0, 0.0, 0.1], [0.0, 1.0, 0.1], [2.0, 1.0, 0.1]]
    out2 = _dump(runner, write_case(str(tmp_path), "flipped", cells=(16, 8, 1), box_hi=(1, 1, 1), vertices=verts,
                                    boundaries=TWO_D))
    assert "mesh curvilinear (trilinear, graded)" in out2
    arc = [(0, 1, (0.0, 1.5, 0.0)), (4, 5, (0.0, 1.5, 1.0))]
    ring = [[1.0, 1.0, 0.0], [-1.0, 1.0, 0.0], [-0.5, 0.5, 0.0], [0.5, 0.5, 0.0],
            [1.0, 1.0, 1.0], [-1.0, 1.0, 1.0], [-0.5, 0.5, 1.0], [0.5, 0.5, 1.0]]
    per = {"Left": "periodic", "Right": "periodic", "sideWalls": "zeroGradient", "frontBack": "empty"}
    r = run(runner, write_case(str(tmp_path), "ring", cells=(20, 10, 1), box_hi=(1, 1, 1), vertices=ring,
                               edges=arc, boundaries=per), "--describe")
    assert r.returncode == 3 and "periodic ends on a graded or curved block" in r.stderr


PIN_BLOCKS = {
    # arc block 1 of createMesh, shortened in z and scaled (edges scale with it)
    "arc": dict(cells=(40, 20, 30), vertices=CREATEMESH["vertices"], hex=CREATEMESH["hex_1"], scale=0.01,
                edges=[(int(a), int(b), p) for (a, b), p in zip(CREATEMESH["edge_vertices"], CREATEMESH["edge_points"])]),
    # the centre box of createMesh, listed against the axes (TFI: the file has edges)
    "centre": dict(cells=(20, 20, 10), vertices=CREATEMESH["vertices"], hex=CREATEMESH["hex_0"],
                   edges=[(int(a), int(b), p) for (a, b), p in zip(CREATEMESH["edge_vertices"],
                                                                  CREATEMESH["edge_points"])]),
    "graded": dict(cells=(12, 8, 6), vertices=[[-0.5, 0.25, 1.0], [1.5, 0.25, 1.0], [1.5, 1.0, 1.0], [-0.5, 1.0, 1.0],
                                               [-0.5, 0.25, 1.6], [1.5, 0.25, 1.6], [1.5, 1.0, 1.6], [-0.5, 1.0, 1.6]],
                   grading=(2.0, 0.5, 1.3)),
    "skewed": dict(cells=(14, 9, 7), grading=(1.2, 0.9, 1.1),
                   vertices=[[0, 0, 0], [1.2, 0.15, 0.1], [1.35, 0.95, -0.05], [-0.1, 0.8, 0], [0.05, 0.02, 0.5],
                             [1.1, 0.2, 0.6], [1.3, 1.0, 0.55], [0, 0.9, 0.45]]),
}


@pytest.mark.parametrize("name", sorted(PIN_BLOCKS))
def test_block_geometry_is_the_reference_generators(runner, tmp_path, name):
    """The host's node coordinates equal, bit for bit, those of the
    reference's own generator compiled from its sources (oracle/_ref), for
    arc-edged, graded and skewed blocks; the metrics handed to the provider
    equal, bit for bit, the oracle's restatement of the reference Field's
    metrics from those coordinates (ghost extrapolation, symmetric
    conservative cofactors, outer-layer copies), with the same identity
    residual."""
    import pyoracle as po
    if po.ref_mesh_lib() is None:
        pytest.skip("oracle/_ref/libsfmesh.so not built (reference sources unavailable)")
    kw = PIN_BLOCKS[name]
    d = write_case(str(tmp_path), name, box_hi=(1, 1, 1), boundaries=ALL_ZG, **kw)
    fp, fm = os.path.join(d, "p.bin"), os.path.join(d, "m.bin")
    out = _dump(runner, d, "--dump-points", fp, "--dump-metrics", fm)
    c = kw["cells"]
    P = np.fromfile(fp).reshape(c[2] + 1, c[1] + 1, c[0] + 1, 3)
    R = po.ref_mesh_points(kw["vertices"], kw.get("hex", range(8)), c, kw.get("grading", (1.0, 1.0, 1.0)),
                           kw.get("edges", ()), kw.get("scale", 1.0))
    assert np.array_equal(P, R)
    want, res, tol = po.field_metrics(R, 3)
    assert np.array_equal(np.fromfile(fm).reshape(want.shape), want)
    line = out.split("metric identity residual ")[1].splitlines()[0]
    assert float(line.split(",")[0]) == float("%.3g" % res) and res <= tol


def test_batch_mode_groups_cases_and_reports_the_rest(runner, tmp_path):
    """`sfg_run --batch` groups case directories by time recipe (one batch
    each) and reports the cases the batched kernels do not run, without a
    GPU under --describe."""
    a = write_case(str(tmp_path), "a", cells=(200, 1, 1), box_hi=(1.0, 0.1, 0.1))
    b = write_case(str(tmp_path), "b", cells=(30, 20, 1), box_hi=(1.5, 1.0, 0.1), convection="teno5Roe",
                   boundaries={"Left": "zeroGradient", "Right": "zeroGradient", "sideWalls": "zeroGradient",
                               "frontBack": "empty"})
    c = write_case(str(tmp_path), "c", cells=(100, 1, 1), box_hi=(1.0, 0.1, 0.1), convection="weno7Rusanov",
                   time="forwardEuler")
    d = write_case(str(tmp_path), "d", cells=(100, 1, 1), box_hi=(1.0, 0.1, 0.1), convection="weno5LaxFriedrichs")
    e = write_case(str(tmp_path), "e", cells=(8, 8, 8), box_hi=(1, 1, 1), boundaries=ALL_ZG)
    r = run(runner, "--batch", a, b, c, d, e, "--describe")
    assert r.returncode == 3, r.stdout + r.stderr
    assert "batch time=SSPRK3 cases=2: a(weno5Rusanov) b(teno5Roe)" in r.stdout
    assert "batch time=forwardEuler cases=1: c(weno7Rusanov)" in r.stdout
    assert "d: convection 'weno5LaxFriedrichs': the batched kernels provide Rusanov and Roe faces" in r.stderr
    assert "e: 3-D grids run on single-grid solvers only" in r.stderr
    r2 = run(runner, "--batch", a, c, "--describe")
    assert r2.returncode == 0
