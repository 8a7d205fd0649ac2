"""Generates the golden fixtures in this directory (run where the reference
source tree and oracle/_ref are available: ``python tests/golden/make_golden.py``).

* sod_weno7_t0p2.json -- the reference's frozen WENO7 + Rusanov + forwardEuler
  Sod baseline (test/Sod/sodCase_weno7_t0p2/baseline.json and the case
  parameters of its case directory: 100 x 20 cells on [0,100] x [0,20],
  dz = 0.1, nGhost 4, rho 1 / 0.125, p 1e5 / 1e4, CFL 0.5, writeInterval
  0.05, t = 0.2, zeroGradient Right and sideWalls, no law on Left).
* ref_rhs.npz -- residuals of the reference's own spatial operator
  (SF::divDispatch + Math::spatialResidual, run through oracle/_ref) on small
  seeded states, every provided recipe, 1-D / 2-D / 3-D, transmissive and
  periodic ends.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

REF_CASE = "/root/reference/test/Sod/sodCase_weno7_t0p2"


def sod_fixture():
    with open(os.path.join(REF_CASE, "baseline.json")) as f:
        base = json.load(f)
    out = {
        "source": "sonicSolver test/Sod/sodCase_weno7_t0p2/baseline.json",
        "case": {"cells": [100, 20, 1], "nodes": [101, 21, 2], "length": [100.0, 20.0, 0.1], "n_ghost": 4,
                 "left": {"rho": 1.0, "u": 0.0, "p": 100000.0}, "right": {"rho": 0.125, "u": 0.0, "p": 10000.0},
                 "split_node": 50, "gamma": 1.4, "cfl": 0.5, "write_interval": 0.05, "t_end": 0.2,
                 "recipe": "weno7Rusanov", "time": "forwardEuler",
                 "bc": {"x_lo": "none (ghosts keep initial values, boundary node advanced)",
                        "x_hi": "zeroGradient", "y": "zeroGradient", "z": "empty"}},
        "baseline": base,
    }
    with open(os.path.join(HERE, "sod_weno7_t0p2.json"), "w") as f:
        json.dump(out, f, indent=1)


def ref_rhs_fixture():
    import pyoracle as po
    from helpers import NG_OF, smooth_state

    arrays = {}
    grids = [(1, (23, 1, 1), (0.05, 1.0, 1.0)), (2, (13, 11, 1), (0.07, 0.09, 1.0)), (3, (7, 6, 5), (0.1, 0.11, 0.12))]
    recipes = [("weno5", po.WENO5, "Rusanov", po.RUSANOV), ("weno5", po.WENO5, "Roe", po.ROE),
               ("teno5", po.TENO5, "Rusanov", po.RUSANOV), ("teno5", po.TENO5, "Roe", po.ROE),
               ("weno3", po.WENO3, "Rusanov", po.RUSANOV), ("weno7", po.WENO7, "Rusanov", po.RUSANOV)]
    for gi, (dim, n, h) in enumerate(grids):
        for bc in (po.BC_TRANSMISSIVE, po.BC_PERIODIC):
            for shock in ((True,) if dim == 3 else (False, True)):
                q = smooth_state(dim, n, seed=11 + gi, shock=shock)
                state = f"{dim}d_bc{bc}_{'shock' if shock else 'smooth'}"
                arrays[state + "_q"] = q
                arrays[state + "_h"] = np.array(h)
                for sname, scheme, fname, flux in recipes:
                    spec = po.GridSpec(dim=dim, n=n, ng=NG_OF[sname], h=h, bc_lo=(bc,) * 3, bc_hi=(bc,) * 3)
                    Q = spec.empty()
                    spec.interior(Q)[...] = q
                    po.fill_ghosts(spec, Q)
                    R = po.RefCase(spec, scheme, flux).rhs(Q)
                    arrays[f"{state}_{sname}{fname}_r"] = np.ascontiguousarray(spec.interior(R))
    np.savez_compressed(os.path.join(HERE, "ref_rhs.npz"), **arrays)


if __name__ == "__main__":
    sod_fixture()
    ref_rhs_fixture()
    print("fixtures written to", HERE)
