"""Shared helpers of the parity tests: node arrays <-> oracle compact arrays,
seeded test states."""
from __future__ import annotations

import numpy as np

import pyoracle as po
from sonicsolver_b200 import capi, cases

SCHEME_OF = {"weno3": po.WENO3, "weno5": po.WENO5, "teno5": po.TENO5, "weno7": po.WENO7}
FLUX_OF = {"Steger": po.STEGER, "Rusanov": po.RUSANOV, "LaxFriedrichs": po.LAXFRIEDRICHS, "Roe": po.ROE,
           "LaxWendroff": po.LAXWENDROFF}
TIME_OF = {"forwardEuler": po.EULER, "SSPRK3": po.SSPRK3, "classicalRK4": po.RK4}
NG_OF = {"weno3": 2, "weno5": 3, "teno5": 3, "weno7": 4}


def split_recipe(recipe: str):
    for s in SCHEME_OF:
        if recipe.startswith(s):
            return s, recipe[len(s):]
    raise ValueError(recipe)


def oracle_spec(case_or_dim, n=None, h=None, bc_lo=None, bc_hi=None, recipe="weno5Rusanov", gamma=1.4):
    if isinstance(case_or_dim, cases.Case):
        c = case_or_dim
        dim, n, h, bc_lo, bc_hi, gamma = c.dim, c.n, c.h, c.bc_lo, c.bc_hi, c.gamma
    else:
        dim = case_or_dim
    scheme, _ = split_recipe(recipe)
    return po.GridSpec(dim=dim, n=tuple(n), ng=NG_OF[scheme], h=tuple(h), bc_lo=tuple(bc_lo), bc_hi=tuple(bc_hi),
                       gamma=gamma)


def to_oracle(spec: po.GridSpec, q_nodes: np.ndarray) -> np.ndarray:
    Q = spec.empty()
    spec.interior(Q)[...] = q_nodes.reshape(spec.interior(Q).shape)
    po.fill_ghosts(spec, Q)
    return Q


def from_oracle(spec: po.GridSpec, Q: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(spec.interior(Q))


def smooth_state(dim, n, seed=0, amp=0.2, gamma=1.4, shock=False, noise=0.01):
    """A seeded smooth (optionally with a contact/shock jump) positive state,
    with `noise` relative random noise on the density."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = n[2], n[1], n[0]
    z, y, x = np.meshgrid(np.linspace(0, 1, nz, endpoint=False), np.linspace(0, 1, ny, endpoint=False),
                          np.linspace(0, 1, nx, endpoint=False), indexing="ij")
    k = rng.uniform(1, 3, 6)
    ph = rng.uniform(0, 2 * np.pi, 6)
    rho = 1.0 + amp * np.sin(2 * np.pi * (k[0] * x + k[1] * y + k[2] * z) + ph[0])
    u = 0.3 * np.cos(2 * np.pi * k[3] * x + ph[1])
    v = 0.2 * np.sin(2 * np.pi * k[4] * y + ph[2]) if dim > 1 else 0 * x
    w = 0.1 * np.cos(2 * np.pi * k[5] * z + ph[3]) if dim > 2 else 0 * x
    p = 1.0 + amp * np.cos(2 * np.pi * (k[1] * x - k[0] * y) + ph[4])
    if shock:
        # a contact + pressure jump across a slanted plane (kept moderate so
        # the reference accepts every reconstructed state: it exits on p <= 0)
        jump = (x + 0.37 * y + 0.21 * z) > 0.55
        rho = np.where(jump, 0.5 * rho, rho)
        p = np.where(jump, 0.4 * p, p)
    rho = rho * (1 + noise * rng.random(rho.shape))
    return cases.conserved(rho, u, v, w, p, gamma)


def curvilinear_metrics(dim, n, h, ng, amp=0.15, field_layout=False, seed=0):
    """Metrics of the smooth map x = h i + amp h sin(...) of the index space
    (i, j, k), 10 per point as the reference Field holds them: Jac = 1/J with
    J = det(dx/di), and the rows of (dx/di)^-1 (XiX, XiY, XiZ, EtX, ...).
    The displacement is periodic in every index over the node count, so the
    same map serves periodic axes.  Points cover the oracle's compact layout
    (ghosts on active axes), or with `field_layout` the Field layout (ghosts
    on every axis).  Returns an array (mz, my, mx, 10)."""
    rng = np.random.default_rng(seed)
    ph = rng.uniform(0, 2 * np.pi, 6)
    ext = [n[d] + (2 * ng if (d < dim or field_layout) else 0) for d in range(3)]
    off = [ng if (d < dim or field_layout) else 0 for d in range(3)]
    k, j, i = np.meshgrid(np.arange(ext[2]) - off[2], np.arange(ext[1]) - off[1], np.arange(ext[0]) - off[0],
                          indexing="ij")
    tw = [2 * np.pi / n[d] if d < dim else 0.0 for d in range(3)]
    idx = [i, j, k]
    # displacement component c depends on the index of axis (c + 1) % dim
    A = np.zeros(i.shape + (3, 3))
    for c in range(3):
        A[..., c, c] = h[c]
        if c >= dim:
            continue
        o = (c + 1) % dim
        if o == c:
            continue
        A[..., c, o] += amp * h[c] * tw[o] * np.cos(tw[o] * idx[o] + ph[c])
        # and a weak self term so the map stays curved in 1-D
    if dim == 1:
        A[..., 0, 0] = h[0] * (1.0 + 0.3 * amp * np.cos(tw[0] * i + ph[0]))
    J = np.linalg.det(A)
    inv = np.linalg.inv(A)
    out = np.empty(i.shape + (10,))
    out[..., 0] = 1.0 / J
    out[..., 1:10] = inv.reshape(i.shape + (9,))
    return out
