"""sonicsolver_b200 -- B200-native explicit Euler provider for sonicSolver.

The product is the sm_100a shared library ``libsonicsolver_b200.so`` behind the
C ABI ``include/sonicsolver_b200.h``; :mod:`sonicsolver_b200.capi` binds it
from Python and :mod:`sonicsolver_b200.cases` builds the workloads.
"""
from . import capi  # noqa: F401

__all__ = ["capi"]
