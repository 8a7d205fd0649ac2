"""Resuming a run (sfg_restore; `sfg_run --checkpoint / --restart`).

A run stopped between two steps, downloaded, and restored with the time and
step count it had reached (into a new solver of the same grid and numerics)
must continue with the same dt sequence and the same bits as the run that was
never stopped: the device keeps nothing across steps but the state and the
clock, and the CFL minimum of the restored state is recomputed exactly.  The
comparison is bit for bit (np.array_equal), in both precisions, on every
kernel family a single grid can take: the 2-D tile variants and sweeps, the
1-D whole-run cluster kernel, the 3-D path, a curvilinear grid and law ends.
"""
import json
import os
import subprocess

import numpy as np
import pytest

from case_dirs import write_case
from sonicsolver_b200 import capi, cases

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RUNNER = os.path.join(ROOT, "sonicsolver_b200", "sfg_run")


def _law_tube():
    c = cases.sod_1d(cells=300, t_end=0.08)
    c.bc_lo = (capi.BC_LAW, 0, 0)
    c.bc_hi = (capi.BC_LAW, 0, 0)
    return c


def _laws(s):
    s.set_boundary_law(0, 0, capi.LAW_FIXED_VALUE, capi.LAW_FIXED_VALUE, capi.LAW_FIXED_VALUE, rho_value=1.0,
                       velocity_value=(0.3, 0.0, 0.0), pressure_value=1.0)
    s.set_boundary_law(0, 1, capi.LAW_ZERO_GRADIENT, capi.LAW_FIXED_VALUE, capi.LAW_ZERO_GRADIENT)


CASES = {
    "vortex2d": lambda: cases.isentropic_vortex(128, t_end=0.6),
    "sod1d": lambda: cases.sod_1d(cells=400, t_end=0.06),
    "tgv3d": lambda: cases.taylor_green(32, t_end=0.2),
    "wavy2d": lambda: cases.wavy_vortex(96, t_end=0.5),
    "laws1d": _law_tube,
}


def _solver(c, precision, variant):
    s = c.solver(precision=precision)
    if c.bc_lo[0] == capi.BC_LAW:
        _laws(s)
    if variant is not None:
        s.variant = variant
    return s


@pytest.mark.parametrize("precision", [capi.PREC_FP64, capi.PREC_FP32_FLUX])
@pytest.mark.parametrize("name,variant", [("vortex2d", 0), ("vortex2d", 1), ("vortex2d", 2), ("sod1d", None),
                                          ("tgv3d", None), ("wavy2d", None), ("laws1d", None)])
def test_restored_run_continues_bit_for_bit(name, variant, precision):
    c = CASES[name]()
    straight = _solver(c, precision, variant)
    st, _ = straight.advance(c.t_end, graph_steps=8)
    want = straight.download()
    t_want, n_want = straight.time()
    straight.close()
    assert st.status_bits == 0 and n_want > 12

    first = _solver(c, precision, variant)
    first.advance(c.t_end, max_steps=n_want // 2, graph_steps=8)
    mid = first.download()
    t_mid, n_mid = first.time()
    first.close()
    assert n_mid == n_want // 2 and t_mid < t_want

    resumed = _solver(c, precision, variant)
    resumed.restore(mid, t_mid, n_mid)
    assert resumed.time() == (t_mid, n_mid)
    st2, _ = resumed.advance(c.t_end, graph_steps=8)
    got = resumed.download()
    assert resumed.time() == (t_want, n_want) and st2.status_bits == 0
    resumed.close()
    assert np.array_equal(got, want)


def test_restore_arguments_are_checked():
    c = cases.sod_1d(cells=50)
    s = c.solver()
    q = np.ascontiguousarray(c.q)
    with pytest.raises(capi.SolverError):
        s.restore(q, float("nan"), 3)
    with pytest.raises(capi.SolverError):
        s.restore(q, 0.1, -1)
    s.restore(q, 0.25, 7)
    assert s.time() == (0.25, 7)
    s.close()


LAW_CASE = {
    "Left": {"rho": "fixedValue: 1.0", "U": "fixedValue: [0.3 0 0]", "p": "fixedValue: 1.0"},
    "Right": {"rho": "zeroGradient", "U": "noSlip", "p": "zeroGradient"},
    "sideWalls": "empty", "frontBack": "empty",
}


def _run(d, *args):
    r = subprocess.run([RUNNER, d, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1]), r.stdout


@pytest.mark.parametrize("mode", ["graph", "plan"])
def test_restart_file_continues_the_case(tmp_path, mode):
    """sfg_run writes a restart file at every output time; a run restarted
    from the first one ends on the bits, the step count and the output
    numbering of the run that wrote it (a 2-D box with an inflow law, a wall
    and zeroGradient side walls, three output times)."""
    bnd = dict(LAW_CASE, sideWalls="zeroGradient")
    d = write_case(str(tmp_path), "ck", cells=(96, 24, 1), box_hi=(1.0, 0.25, 0.1), end_time=0.09375,
                   write_interval=0.03125, boundaries=bnd)
    prefix = os.path.join(d, "restart")
    s1, out1 = _run(d, "--mode", mode, "--checkpoint", prefix, "--dump", os.path.join(d, "a.bin"))
    assert s1["status"] == 0 and s1["outputs"] == 3
    for k in range(3):
        assert os.path.exists(f"{prefix}_{k:04d}.json")
    assert os.path.exists(prefix + "_end.json")
    with open(prefix + "_0000.json") as f:
        doc = json.load(f)
    assert doc["formatVersion"] == 1 and doc["outputs"] == 1 and doc["nextOutput"] == 0.0625
    assert set(doc["fields"]) == {"rho", "rhoU", "rhoE"} and doc["fields"]["rhoU"]["size"] == 97 * 25
    s2, out2 = _run(d, "--mode", mode, "--restart", prefix + "_0000.json", "--dump", os.path.join(d, "b.bin"))
    assert "restart t=0.03125" in out2
    assert s2["steps"] == s1["steps"] and s2["time"] == s1["time"] and s2["outputs"] == 3
    assert np.array_equal(np.fromfile(os.path.join(d, "b.bin")), np.fromfile(os.path.join(d, "a.bin")))
    # the restarted run wrote the later outputs under their own numbers
    assert "_0001.vts" in out2 and "_0000.vts" not in out2


def test_restart_file_errors(tmp_path):
    d = write_case(str(tmp_path), "bad", cells=(40, 1, 1), box_hi=(1.0, 0.1, 0.1), end_time=0.02)
    prefix = os.path.join(d, "r")
    _run(d, "--no-write", "--checkpoint", prefix)
    with open(prefix + "_end.json") as f:
        doc = json.load(f)
    doc["fields"]["rho"]["values"] = doc["fields"]["rho"]["values"][:-1]
    with open(os.path.join(d, "short.json"), "w") as f:
        json.dump(doc, f)
    r = subprocess.run([RUNNER, d, "--restart", os.path.join(d, "short.json")], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 1 and "incompatible field rho" in r.stderr
    d2 = write_case(str(tmp_path), "other", cells=(50, 1, 1), box_hi=(1.0, 0.1, 0.1), end_time=0.02)
    r2 = subprocess.run([RUNNER, d2, "--restart", prefix + "_end.json"], capture_output=True, text=True, timeout=120)
    assert r2.returncode == 1 and "holds 41 x 1 x 1 nodes" in r2.stderr
