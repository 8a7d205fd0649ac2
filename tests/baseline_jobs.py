"""Oracle runs of the benchmark workloads at their full sizes, for the GPU
parity tests in test_gpu_baseline_sizes.py.

Each job is a plain function of picklable arguments, so the tests run them in
a process pool (spawn context: the workers never touch CUDA) while the GPU
side of the same tests runs.  Every job builds its own initial state from the
case generators, so the arrays that cross processes are results only.
"""
from __future__ import annotations

import numpy as np

import pyoracle as po
from helpers import FLUX_OF, SCHEME_OF, TIME_OF, from_oracle, oracle_spec, split_recipe, to_oracle
from sonicsolver_b200 import cases

TUBE_SEED = 2024   # the batched shock-tube workload: 512 tubes from this seed
TUBE_COUNT = 512


def _ids(recipe, time_recipe):
    scheme, flux = split_recipe(recipe)
    return SCHEME_OF[scheme], FLUX_OF[flux], TIME_OF[time_recipe]


def oracle_steps(case: cases.Case, steps: int, keep=()):
    """The oracle's Time::Driver loop (CFL dt every step) for `steps` steps
    of `case`.  Returns (dts, states) with the node state after each step
    number listed in `keep` (and always after the last)."""
    spec = oracle_spec(case, recipe=case.recipe)
    scheme, flux, time_id = _ids(case.recipe, case.time_recipe)
    Q = to_oracle(spec, case.q)
    dts, states, t = [], {}, 0.0
    for k in range(1, steps + 1):
        d, t = po.advance(spec, scheme, flux, time_id, Q, case.t_end, case.cfl, t_start=t, max_steps=1)
        dts.extend(d.tolist())
        if k in keep or k == steps:
            states[k] = from_oracle(spec, Q).copy()
    return np.array(dts), states


def vortex_1024_steps(steps=5):
    """The 2-D periodic isentropic vortex, 1024^2 cells, TENO5 + Rusanov,
    SSPRK3, CFL 0.4: states after step 1 and after `steps` steps."""
    return oracle_steps(cases.isentropic_vortex(1024), steps, keep=(1,))


def taylor_green_steps(N=128, steps=1):
    """Taylor-Green vortex N^3, WENO5 + Rusanov, SSPRK3, CFL 0.5."""
    return oracle_steps(cases.taylor_green(N), steps)


def taylor_green_planes(N, zs):
    """The Taylor-Green initial state on the z-planes `zs` only (the same
    expressions as cases.taylor_green, evaluated per plane)."""
    full_h = 2 * np.pi / N
    x = np.arange(N) * full_h
    z = x[np.asarray(zs) % N]
    Z, Y, X = np.meshgrid(z, x, x, indexing="ij")
    gamma, mach = 1.4, 0.1
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    p0 = 1.0 / (gamma * mach * mach)
    p = p0 + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    return cases.conserved(np.ones_like(X), u, v, 0.0, p, gamma)


def taylor_green_slab_residual(N, z0, m, recipe="weno5Rusanov"):
    """The oracle residual of the periodic Taylor-Green state on planes
    z0 .. z0+m-1 (mod N), from a slab that carries their periodic halo:
    planes z0-4 .. z0+m+3.  Only the middle m planes are returned.  Their
    stencils reach 3 planes out; the slab's own z ends are transmissive
    boundary nodes, which the oracle replaces by their inner neighbours, so
    the halo is one plane deeper than the stencil and the ends never enter."""
    halo = 4
    zs = np.arange(z0 - halo, z0 + m + halo)
    q = taylor_green_planes(N, zs)
    h = 2 * np.pi / N
    bc_lo, bc_hi = (1, 1, 0), (1, 1, 0)
    spec = oracle_spec(3, (N, N, m + 2 * halo), (h, h, h), bc_lo, bc_hi, recipe)
    scheme, flux, _ = _ids(recipe, "SSPRK3")
    R = from_oracle(spec, po.rhs(spec, scheme, flux, to_oracle(spec, q)))
    return R[halo:halo + m].copy()


def tube_picks():
    """Indices into the seeded batch: the largest 1-D tube, the largest 2-D
    tube, and the 2-D tube whose diaphragm is closest to the diagonal among
    those of at most 160 cells a side."""
    tubes = cases.shock_tube_batch(count=TUBE_COUNT, seed=TUBE_SEED, t_end=0.15)
    one = [i for i, c in enumerate(tubes) if c.dim == 1]
    two = [i for i, c in enumerate(tubes) if c.dim == 2]
    big1 = max(one, key=lambda i: tubes[i].n[0])
    big2 = max(two, key=lambda i: tubes[i].n[0])
    small2 = [i for i in two if tubes[i].n[0] <= 161]
    slant = min(small2, key=lambda i: abs(tubes[i].meta["angle"] - np.pi / 4))
    return big1, big2, slant


def tube_steps(index, steps=20):
    """`steps` oracle steps of tube `index` of the seeded batch."""
    tubes = cases.shock_tube_batch(count=TUBE_COUNT, seed=TUBE_SEED, t_end=0.15)
    return oracle_steps(tubes[index], steps)
