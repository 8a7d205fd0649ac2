"""The C++17 host side (case reader, provider catalogs, plan, driver) on the
CPU: `sfg_run --selftest` checks the catalog and plan rules, `--describe`
reads a case directory, resolves its providers and validates the plan
bindings without touching a GPU."""
import os
import subprocess

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
    TENO5 + Steger-Warming and WENO7 + Rusanov) resolve and plan; every other
    case is reported as not supported by this provider, with its reason."""
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
    for case in ("sodCase", "sodCase_weno7", "sodCase_weno7_t0p2"):
        assert os.path.join("Sod", case) in resolved


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
