"""Initial conditions, exact solutions and grid descriptions of the workloads.

Node-based grids as in sonicSolver (N cells -> N + 1 nodes per active axis with
transmissive ends; N unique nodes x_i = i L / N on periodic axes).  State
arrays are AoS ``[k][j][i][v]`` over the nodes, v = (rho, rho u, rho v, rho w, E).

Workloads (sizes from the project configuration):
  * Sod shock tube, 1-D, 1000 cells;
  * 2-D periodic isentropic vortex on [0, 10]^2;
  * 3-D inviscid Taylor-Green vortex on [0, 2 pi]^3 at Mach 0.1;
  * batched shock tubes (seeded, mixed 1-D / 2-D, uneven sizes).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import capi


@dataclass
class Case:
    name: str
    dim: int
    n: tuple          # nodes per axis
    h: tuple          # spacing per axis
    bc_lo: tuple
    bc_hi: tuple
    q: np.ndarray     # AoS nodes, shape (nz, ny, nx, 5)
    gamma: float = 1.4
    t_end: float = 0.0
    cfl: float = 0.5
    recipe: str = "weno5Rusanov"
    time_recipe: str = "SSPRK3"
    meta: dict = field(default_factory=dict)
    metrics: np.ndarray | None = None   # curvilinear: (nz, ny, nx, 10) per node (sfg_set_metrics)

    @property
    def cells(self) -> int:
        """Cells as counted in the workload definitions (N per active axis)."""
        c = 1
        for d in range(self.dim):
            per = self.bc_lo[d] == capi.BC_PERIODIC
            c *= self.n[d] if per else self.n[d] - 1
        return c

    @property
    def nodes(self) -> int:
        return int(np.prod(self.n))

    def solver(self, precision=capi.PREC_FP64, **kw) -> "capi.Solver":
        s = capi.Solver(self.dim, self.n, self.h, self.bc_lo, self.bc_hi, recipe=kw.pop("recipe", self.recipe),
                        time_recipe=kw.pop("time_recipe", self.time_recipe), precision=precision,
                        gamma=self.gamma, cfl=kw.pop("cfl", self.cfl), **kw)
        if self.metrics is not None:
            s.set_metrics(self.metrics)
        s.upload(np.ascontiguousarray(self.q))
        return s


def conserved(rho, u, v, w, p, gamma=1.4) -> np.ndarray:
    """Primitive -> conserved, stacked on a last axis of length 5."""
    rho = np.asarray(rho, dtype=np.float64)
    shape = np.broadcast(rho, u, v, w, p).shape
    q = np.empty(shape + (5,))
    q[..., 0] = rho
    q[..., 1] = rho * u
    q[..., 2] = rho * v
    q[..., 3] = rho * w
    q[..., 4] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return q


def primitive(q: np.ndarray, gamma=1.4):
    rho = q[..., 0]
    u, v, w = q[..., 1] / rho, q[..., 2] / rho, q[..., 3] / rho
    p = (gamma - 1.0) * (q[..., 4] - 0.5 * rho * (u * u + v * v + w * w))
    return rho, u, v, w, p


# --------------------------------------------------------------------- Sod

def sod_1d(cells=1000, gamma=1.4, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), x_split=0.5,
           recipe="weno5Rusanov", time_recipe="SSPRK3", cfl=0.5, t_end=0.2) -> Case:
    """Sod tube on x in [0, 1]: `cells` cells, transmissive ends.  A node at
    the diaphragm takes the right state (leftHalf holds i < nodes/2 in the
    reference mesh sets, SF_meshGen.cpp:533-541)."""
    n = cells + 1
    x = np.arange(n) / cells
    is_left = x < x_split
    rho = np.where(is_left, left[0], right[0])
    u = np.where(is_left, left[1], right[1])
    p = np.where(is_left, left[2], right[2])
    q = conserved(rho, u, 0.0, 0.0, p, gamma)[None, None]
    return Case("sod1d", 1, (n, 1, 1), (1.0 / cells, 1.0, 1.0), (0, 0, 0), (0, 0, 0), q, gamma, t_end, cfl,
                recipe, time_recipe)


def sod_exact(x, t, gamma=1.4, left=(1.0, 0.0, 1.0), right=(0.125, 0.0, 0.1), x0=0.5):
    """Exact Riemann solution (ideal gas, Toro ch. 4): (rho, u, p) at x, t."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(gamma * pl / rl), math.sqrt(gamma * pr / rr)

    def f(p, rk, pk, ck):
        if p > pk:
            A, B = 2.0 / ((gamma + 1) * rk), (gamma - 1) / (gamma + 1) * pk
            return (p - pk) * math.sqrt(A / (p + B))
        return 2 * ck / (gamma - 1) * ((p / pk) ** ((gamma - 1) / (2 * gamma)) - 1)

    lo, hi = 1e-12, max(pl, pr) * 10
    for _ in range(200):
        pm = 0.5 * (lo + hi)
        if f(pm, rl, pl, cl) + f(pm, rr, pr, cr) + ur - ul > 0:
            hi = pm
        else:
            lo = pm
    ps = 0.5 * (lo + hi)
    us = 0.5 * (ul + ur) + 0.5 * (f(ps, rr, pr, cr) - f(ps, rl, pl, cl))
    g = gamma
    out = np.zeros((3,) + np.shape(x))
    s = (np.asarray(x) - x0) / max(t, 1e-300)
    res = []
    for si in np.ravel(s):
        if si <= us:  # left of contact
            if ps > pl:
                sl = ul - cl * math.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                res.append((rl, ul, pl) if si < sl else (rl * ((ps / pl + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pl + 1)), us, ps))
            else:
                shl = ul - cl
                csl = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - csl
                if si < shl:
                    res.append((rl, ul, pl))
                elif si > stl:
                    res.append((rl * (ps / pl) ** (1 / g), us, ps))
                else:
                    uu = 2 / (g + 1) * (cl + (g - 1) / 2 * ul + si)
                    cc = 2 / (g + 1) * (cl + (g - 1) / 2 * (ul - si))
                    rho = rl * (cc / cl) ** (2 / (g - 1))
                    res.append((rho, uu, pl * (cc / cl) ** (2 * g / (g - 1))))
        else:
            if ps > pr:
                sr = ur + cr * math.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                res.append((rr, ur, pr) if si > sr else (rr * ((ps / pr + (g - 1) / (g + 1)) / ((g - 1) / (g + 1) * ps / pr + 1)), us, ps))
            else:
                shr = ur + cr
                csr = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + csr
                if si > shr:
                    res.append((rr, ur, pr))
                elif si < str_:
                    res.append((rr * (ps / pr) ** (1 / g), us, ps))
                else:
                    uu = 2 / (g + 1) * (-cr + (g - 1) / 2 * ur + si)
                    cc = 2 / (g + 1) * (cr - (g - 1) / 2 * (ur - si))
                    rho = rr * (cc / cr) ** (2 / (g - 1))
                    res.append((rho, uu, pr * (cc / cr) ** (2 * g / (g - 1))))
    arr = np.array(res).T.reshape((3,) + np.shape(x))
    return arr


# ------------------------------------------------------------ isentropic vortex

def vortex_fields(x, y, t=0.0, L=10.0, beta=5.0, gamma=1.4, center=(5.0, 5.0), uinf=(1.0, 1.0)):
    """Isentropic vortex (Shu 1998 form) advected by (uinf) on a periodic box:
    du = -beta/(2 pi) e^{(1-r^2)/2} (y - yc), dv = beta/(2 pi) e^{(1-r^2)/2} (x - xc),
    T = 1 - (gamma-1) beta^2/(8 gamma pi^2) e^{1-r^2}, rho = T^{1/(gamma-1)}, p = rho^gamma."""
    xc = (center[0] + uinf[0] * t) % L
    yc = (center[1] + uinf[1] * t) % L
    dx = (x - xc + 0.5 * L) % L - 0.5 * L
    dy = (y - yc + 0.5 * L) % L - 0.5 * L
    r2 = dx * dx + dy * dy
    e = np.exp(0.5 * (1.0 - r2))
    u = uinf[0] - beta / (2 * math.pi) * e * dy
    v = uinf[1] + beta / (2 * math.pi) * e * dx
    T = 1.0 - (gamma - 1.0) * beta ** 2 / (8.0 * gamma * math.pi ** 2) * e * e
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho ** gamma
    return rho, u, v, p


def isentropic_vortex(N=1024, L=10.0, beta=5.0, gamma=1.4, recipe="teno5Rusanov", time_recipe="SSPRK3",
                      cfl=0.4, t_end=10.0) -> Case:
    h = L / N
    x = np.arange(N) * h
    X, Y = np.meshgrid(x, x, indexing="xy")
    rho, u, v, p = vortex_fields(X, Y, 0.0, L, beta, gamma)
    q = conserved(rho, u, v, 0.0, p, gamma)[None]
    return Case("isentropic_vortex", 2, (N, N, 1), (h, h, 1.0), (1, 1, 0), (1, 1, 0), q, gamma, t_end, cfl,
                recipe, time_recipe, meta={"L": L, "beta": beta})


def vortex_exact(case: Case, t: float) -> np.ndarray:
    if "X" in case.meta:   # curvilinear: the nodes' physical coordinates
        X, Y = case.meta["X"], case.meta["Y"]
    else:
        N = case.n[0]
        h = case.h[0]
        x = np.arange(N) * h
        X, Y = np.meshgrid(x, x, indexing="xy")
    rho, u, v, p = vortex_fields(X, Y, t, case.meta["L"], case.meta["beta"], case.gamma)
    return conserved(rho, u, v, 0.0, p, case.gamma)[None]


def wavy_vortex(N=1024, L=10.0, amp=0.3, beta=5.0, gamma=1.4, recipe="teno5Rusanov", time_recipe="SSPRK3",
                cfl=0.4, t_end=10.0) -> Case:
    """The isentropic vortex on a sheared periodic mesh: node (i, j) sits at
    x = i h + A sin(2 pi j / N), y = j h + A sin(2 pi i / N), A = amp L / (2 pi)
    (amp < 1 keeps the map invertible).  Metrics are the map's exact ones
    with respect to the node index: Jac = 1 / det(dx/di), the xi / eta / zeta
    vectors the rows of (dx/di)^-1; the z slab is 1 thick."""
    h = L / N
    A = amp * L / (2 * math.pi)
    i = np.arange(N)
    I, J = np.meshgrid(i, i, indexing="xy")
    k = 2 * math.pi / N
    X = I * h + A * np.sin(k * J)
    Y = J * h + A * np.sin(k * I)
    dxdj = A * k * np.cos(k * J)
    dydi = A * k * np.cos(k * I)
    det = h * h - dxdj * dydi      # times the slab thickness 1
    M = np.zeros((1, N, N, 10))
    M[0, ..., 0] = 1.0 / det
    M[0, ..., 1] = h / det         # xi_x, xi_y (inverse of [[h, dxdj], [dydi, h]])
    M[0, ..., 2] = -dxdj / det
    M[0, ..., 4] = -dydi / det     # eta_x, eta_y
    M[0, ..., 5] = h / det
    M[0, ..., 9] = 1.0             # zeta_z
    rho, u, v, p = vortex_fields(X, Y, 0.0, L, beta, gamma)
    q = conserved(rho, u, v, 0.0, p, gamma)[None]
    return Case("wavy_vortex", 2, (N, N, 1), (h, h, 1.0), (1, 1, 0), (1, 1, 0), q, gamma, t_end, cfl, recipe,
                time_recipe, meta={"L": L, "beta": beta, "amp": amp, "X": X, "Y": Y}, metrics=M)


# ------------------------------------------------------------ Taylor-Green

def taylor_green(N=256, mach=0.1, gamma=1.4, recipe="weno5Rusanov", time_recipe="SSPRK3", cfl=0.5,
                 t_end=10.0) -> Case:
    """Inviscid compressible Taylor-Green vortex on [0, 2 pi]^3, rho = 1,
    p = p0 + (cos 2x + cos 2y)(cos 2z + 2)/16 with p0 = 1/(gamma Ma^2)."""
    L = 2 * math.pi
    h = L / N
    x = np.arange(N) * h
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    p0 = 1.0 / (gamma * mach * mach)
    p = p0 + (np.cos(2 * X) + np.cos(2 * Y)) * (np.cos(2 * Z) + 2.0) / 16.0
    q = conserved(np.ones_like(X), u, v, 0.0, p, gamma)
    return Case("taylor_green", 3, (N, N, N), (h, h, h), (1, 1, 1), (1, 1, 1), q, gamma, t_end, cfl, recipe,
                time_recipe, meta={"mach": mach})


def kinetic_energy(q: np.ndarray) -> float:
    return float(0.5 * np.sum((q[..., 1] ** 2 + q[..., 2] ** 2 + q[..., 3] ** 2) / q[..., 0]))


# ------------------------------------------------------------ batched shock tubes

def shock_tube_batch(count=512, seed=2024, gamma=1.4, recipe="weno5Rusanov", time_recipe="SSPRK3",
                     cfl=0.5, t_end=0.15, max_1d=16384, max_2d=512):
    """Seeded batch of independent shock tubes: half 1-D (cells log-uniform
    in [256, max_1d]), half 2-D (side log-uniform in [64, max_2d], diaphragm
    through the centre at an angle uniform in [0, pi)); rho, p log-uniform in
    [0.1, 10] per side, u uniform in [-1, 1]; unit domain, transmissive ends."""
    rng = np.random.default_rng(seed)
    cases = []
    for b in range(count):
        two_d = b >= count // 2
        rl, rr, pl, pr = np.exp(rng.uniform(math.log(0.1), math.log(10.0), 4))
        ul, ur = rng.uniform(-1.0, 1.0, 2)
        if not two_d:
            cells = int(round(math.exp(rng.uniform(math.log(256), math.log(max_1d)))))
            c = sod_1d(cells, gamma, (rl, ul, pl), (rr, ur, pr), 0.5, recipe, time_recipe, cfl, t_end)
            c.name = f"tube1d_{b}"
        else:
            side = int(round(math.exp(rng.uniform(math.log(64), math.log(max_2d)))))
            ang = rng.uniform(0.0, math.pi)
            n = side + 1
            x = np.arange(n) / side
            X, Y = np.meshgrid(x, x, indexing="xy")
            s = (X - 0.5) * math.cos(ang) + (Y - 0.5) * math.sin(ang)
            left = s < 0
            nx_, ny_ = math.cos(ang), math.sin(ang)
            rho = np.where(left, rl, rr)
            un = np.where(left, ul, ur)
            p = np.where(left, pl, pr)
            q = conserved(rho, un * nx_, un * ny_, 0.0, p, gamma)[None]
            c = Case(f"tube2d_{b}", 2, (n, n, 1), (1.0 / side, 1.0 / side, 1.0), (0, 0, 0), (0, 0, 0), q, gamma,
                     t_end, cfl, recipe, time_recipe, meta={"angle": ang})
        c.meta.update({"left": (rl, ul, pl), "right": (rr, ur, pr)})
        cases.append(c)
    return cases
