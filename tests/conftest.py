import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a library")


def rel_linf(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Relative L-infinity error per conserved variable: max|a-b| / max|b|
    over the field (a variable that is identically zero in b is scaled by the
    largest variable scale)."""
    a = np.asarray(a).reshape(-1, 5)
    b = np.asarray(b).reshape(-1, 5)
    scale = np.abs(b).max(axis=0)
    floor = scale.max() if scale.max() > 0 else 1.0
    scale = np.where(scale > 0, scale, floor)
    return np.abs(a - b).max(axis=0) / scale


def state_scale(q):
    """Per conserved variable max |q|, one scale for the momentum vector (the
    largest |component| over the three)."""
    scale = np.abs(np.asarray(q).reshape(-1, 5)).max(axis=0)
    scale[1:4] = scale[1:4].max()
    return np.where(scale > 0, scale, 1.0)


def rel_linf_vec(a, b):
    """Relative L-infinity per conserved variable, the momentum components
    measured against one scale (a component that is zero up to round-off,
    such as rho v of a flow along x, is not compared with its own noise)."""
    a = np.asarray(a).reshape(-1, 5)
    b = np.asarray(b).reshape(-1, 5)
    return np.abs(a - b).max(axis=0) / state_scale(b)


@pytest.fixture(scope="session")
def oracle():
    import pyoracle
    pyoracle.oracle_lib()
    return pyoracle
