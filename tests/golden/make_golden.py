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
* ref_laws.npz -- the reference's own physical boundary laws
  (Boundary::update for density and velocity, updateEnergyFromPressure; run
  through oracle/_ref `sfr_fill_laws`) applied to small seeded states with
  law ends on every active axis: every density / velocity / pressure law
  combination on a 1-D grid, a cycle of combinations on 2-D and 3-D grids.
* createmesh_blocks.npz -- the reference generator's node coordinates of
  blocks 0, 1 and 2 of its test/createMesh case (block 0: a 40 x 40 x 190
  box whose hex runs against the axes; blocks 1 and 2: 40 x 20 x 190 hexes
  with two arc edges each, transfinite interpolation), read from the
  mesh_block00N.vts files that case holds, on the z planes k = 0, 1, 95,
  190; with the vertices, hexes, cells, grading and arc edges of its
  mesh/generation.yaml.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

# the reference tree, read in place (SONICSOLVER_REFERENCE overrides its location)
REF_ROOT = os.environ.get("SONICSOLVER_REFERENCE", "/root/reference")
REF_CASE = os.path.join(REF_ROOT, "test", "Sod", "sodCase_weno7_t0p2")


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


LAW_GRIDS = [(1, (9, 1, 1)), (2, (8, 7, 1)), (3, (5, 4, 4))]


def law_state(spec, rng):
    """Positive random state on every storage position (ghosts included: the
    laws read the previous ghost and boundary values)."""
    Q = spec.empty()
    Q[..., 0] = rng.uniform(0.5, 2.0, Q.shape[:-1])
    for d in range(3):
        Q[..., 1 + d] = rng.uniform(-0.3, 0.3, Q.shape[:-1]) * Q[..., 0]
    ke = 0.5 * (Q[..., 1] ** 2 + Q[..., 2] ** 2 + Q[..., 3] ** 2) / Q[..., 0]
    Q[..., 4] = rng.uniform(0.5, 2.0, Q.shape[:-1]) / 0.4 + ke
    return Q


def law_specs():
    """(name, GridSpec) of the ref_laws cases."""
    import itertools
    import pyoracle as po
    kinds = [po.LAW_ZERO_GRADIENT, po.LAW_FIXED_VALUE, po.LAW_SYMMETRY]
    combos = list(itertools.product(kinds, kinds, kinds))
    out = []
    for dim, n in LAW_GRIDS:
        use = combos if dim == 1 else combos[::3] if dim == 2 else combos[1::13]
        for combo in use:
            laws = {}
            for d in range(dim):
                for e in (0, 1):
                    laws[(d, e)] = po.LawSpec(*combo, rho_value=1.3 + 0.1 * d, U_value=(0.2 * e, -0.1, 0.05 * d),
                                              p_value=2.2 + 0.2 * e)
            bc = tuple(po.BC_LAW if d < dim else po.BC_TRANSMISSIVE for d in range(3))
            spec = po.GridSpec(dim=dim, n=n, h=(0.1, 0.1, 0.1), bc_lo=bc, bc_hi=bc, laws=laws)
            out.append((f"{dim}d_{combo[0]}{combo[1]}{combo[2]}", spec))
    return out


def ref_laws_fixture():
    import pyoracle as po
    rng = np.random.default_rng(2024)
    arrays = {}
    for name, spec in law_specs():
        Q = law_state(spec, rng)
        out = Q.copy()
        po.ref_fill_laws(spec, out)
        arrays[name + "_in"] = Q
        arrays[name + "_out"] = out
    np.savez_compressed(os.path.join(HERE, "ref_laws.npz"), **arrays)


def createmesh_fixture(blocks=(0, 1, 2), planes=(0, 1, 95, 190)):
    import re
    case = os.path.join(REF_ROOT, "test", "createMesh", "mesh")
    with open(os.path.join(case, "generation.yaml")) as f:
        gen = json.load(f)
    assert all(e["type"] == "arc" for e in gen["edges"])
    out = {"vertices": np.array(gen["vertices"], dtype=np.float64), "planes": np.array(planes),
           "scale": np.array(gen.get("scale", 1.0)),
           "edge_vertices": np.array([e["vertices"] for e in gen["edges"]]),
           "edge_points": np.array([e["point"] for e in gen["edges"]], dtype=np.float64)}
    for b in blocks:
        blk = gen["blocks"][b]
        with open(os.path.join(case, f"mesh_block{b:03d}.vts")) as f:
            text = f.read()
        ext = [int(x) for x in re.search(r'WholeExtent="([^"]+)"', text).group(1).split()]
        nx, ny, nz = ext[1] + 1, ext[3] + 1, ext[5] + 1
        body = re.search(r"<Points>\s*<DataArray[^>]*>(.*?)</DataArray>", text, re.S).group(1)
        pts = np.array(body.split(), dtype=np.float64).reshape(nz, ny, nx, 3)
        assert (nx - 1, ny - 1, nz - 1) == tuple(blk["cells"])
        out[f"points_{b}"] = pts[list(planes)]
        out[f"hex_{b}"] = np.array(blk["vertices"])
        out[f"cells_{b}"] = np.array(blk["cells"])
        out[f"grading_{b}"] = np.array(blk["grading"], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, "createmesh_blocks.npz"), **out)


if __name__ == "__main__":
    sod_fixture()
    ref_rhs_fixture()
    ref_laws_fixture()
    createmesh_fixture()
    print("fixtures written to", HERE)
