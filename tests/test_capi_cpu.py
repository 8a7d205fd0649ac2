"""C-ABI checks that need no GPU: the library loads, exports every entry
point include/sonicsolver_b200.h declares, and refuses to run without a
device (no CPU fallback)."""
import ctypes
import os
import re

import numpy as np
import pytest

from sonicsolver_b200 import capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names |= set(re.findall(r"\b(sfg_\w+)\s*\(", text))
    return names


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    names = declared_symbols()
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(capi.EXPORTS) <= names


def test_recipe_names_round_trip():
    lib = capi.lib()
    for name, rid in capi.RECIPES.items():
        assert lib.sfg_recipe_name(rid).decode() == name
        out = ctypes.c_int()
        assert lib.sfg_recipe_from_name(name.encode(), ctypes.byref(out)) == 0
        assert out.value == rid
    out = ctypes.c_int()
    assert len(capi.RECIPES) == 20
    assert lib.sfg_recipe_from_name(b"primitiveUpwind1", ctypes.byref(out)) == capi.ERR_ARG


def test_invalid_descriptors_rejected_before_device_use():
    with pytest.raises(capi.SolverError) as e:
        capi.Solver(2, (2, 9, 1), (0.1, 0.1, 1.0), (0, 0, 0), (0, 0, 0))
    assert e.value.code == capi.ERR_ARG
    with pytest.raises(capi.SolverError):
        capi.Solver(2, (9, 9, 1), (0.1, 0.1, 1.0), (1, 0, 0), (0, 0, 0))  # periodic on one end only
    with pytest.raises(capi.SolverError):
        capi.Solver(1, (9, 2, 1), (0.1, 0.1, 1.0), (0, 0, 0), (0, 0, 0))  # inactive axis with 2 nodes
    with pytest.raises(capi.SolverError):
        capi.Solver(1, (9, 1, 1), (0.1, 1.0, 1.0), (0, 0, 0), (0, 0, 0), recipe=5)  # weno5Steger not provided


def test_no_cpu_fallback_without_device():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(capi.SolverError) as e:
        capi.Solver(1, (9, 1, 1), (0.1, 1.0, 1.0), (0, 0, 0), (0, 0, 0))
    assert e.value.code == capi.ERR_CUDA


@pytest.mark.parametrize("n,gamma,h", [
    ((1 << 22, 1 << 21, 1 << 21), 1.4, (0.1, 0.1, 0.1)),   # product wraps a signed 64-bit count to 0
    ((70000, 70000, 3), 1.4, (0.1, 0.1, 0.1)),             # each axis below the cap, the product above it
    ((16, 16, 16), float("inf"), (0.1, 0.1, 0.1)),
    ((16, 16, 16), 1.4, (0.1, float("inf"), 0.1)),
])
def test_noalloc_arguments_rejected_before_any_launch(n, gamma, h):
    """sfg_residual_noalloc checks every size against its fixed working array
    (without overflowing the node count) and refuses non-finite gamma or
    spacing, all before it touches the device: the pointers here are never
    dereferenced."""
    with pytest.raises(capi.SolverError) as e:
        capi.residual_noalloc(3, n, h, (1, 1, 1), (1, 1, 1), 4096, 8192, gamma=gamma)
    assert e.value.code == capi.ERR_ARG
