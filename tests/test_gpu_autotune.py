"""Autotuner: picks a valid variant, caches it, and tuning does not change
FP64 results beyond round-off (the variants compute the same operator)."""
import numpy as np
import pytest

from conftest import rel_linf
from sonicsolver_b200 import autotune, capi, cases

pytestmark = pytest.mark.gpu


def test_tune_solver_selects_and_caches(tmp_path, monkeypatch):
    monkeypatch.setenv("SFG_TUNING_FILE", str(tmp_path / "tuning.json"))
    c = cases.isentropic_vortex(160, recipe="teno5Rusanov")
    s = c.solver()
    entry = autotune.tune_solver(s, "teno5Rusanov", capi.PREC_FP64, repeats=2)
    assert entry["best"] in (0, 1, 2) and s.variant == entry["best"]
    assert set(entry["ms_per_stage"]) == {"0", "1", "2"}
    assert (tmp_path / "tuning.json").exists()
    s2 = c.solver()
    again = autotune.tune_solver(s2, "teno5Rusanov", capi.PREC_FP64)
    assert again["best"] == entry["best"] and s2.variant == entry["best"]


def test_variants_give_the_same_fp64_step():
    c = cases.isentropic_vortex(96, recipe="weno5Rusanov")
    out = []
    for v in (0, 1, 2):
        s = c.solver()
        s.variant = v
        s.advance(1e30, max_steps=5)
        out.append(s.download().reshape(c.q.shape))
    assert rel_linf(out[1], out[0]).max() <= 1e-13
    assert rel_linf(out[2], out[0]).max() <= 1e-13


def test_tune_batch(tmp_path, monkeypatch):
    monkeypatch.setenv("SFG_TUNING_FILE", str(tmp_path / "tuning.json"))
    tubes = cases.shock_tube_batch(count=8, seed=1, max_1d=1200, max_2d=128)
    best = autotune.tune_batch(lambda: capi.Batch(1 << 30, 16), tubes, "weno5Rusanov", capi.PREC_FP64, steps=3)
    assert best in (1, 2)
