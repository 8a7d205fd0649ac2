"""ctypes bindings of the CPU checker libraries (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  It wraps

  * oracle/liboracle.so      -- the plain-C restatement (sf_oracle.c);
  * oracle/_ref/libsfref.so  -- the reference translation units driven by
                                ref_driver.cpp (present when the reference
                                sources were available at build time).

Arrays use the oracle's compact node layout: AoS ``[k][j][i][v]`` with ``ng``
ghost layers on active axes only (see sf_oracle.h).
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

WENO3, WENO5, TENO5, WENO7 = 0, 1, 2, 3
STEGER, RUSANOV, LAXFRIEDRICHS, ROE, LAXWENDROFF = 0, 1, 2, 3, 4
EULER, SSPRK3, RK4 = 0, 1, 2
BC_TRANSMISSIVE, BC_PERIODIC, BC_FROZEN, BC_LAW = 0, 1, 2, 3
LAW_ZERO_GRADIENT, LAW_FIXED_VALUE, LAW_SYMMETRY = 0, 1, 2
ERRORS = {0: "ok", 1: "non-finite", 2: "invalid state", 3: "TENO all-cutoff", 4: "argument",
          5: "Roe sound speed"}


class Law(ctypes.Structure):
    """``sfo_law``: density / velocity / pressure law of one LAW end."""
    _fields_ = [("rho", ctypes.c_int), ("U", ctypes.c_int), ("p", ctypes.c_int), ("pad", ctypes.c_int),
                ("rho_value", ctypes.c_double), ("U_value", ctypes.c_double * 3),
                ("p_value", ctypes.c_double)]


class Grid(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n", ctypes.c_int * 3), ("ng", ctypes.c_int),
                ("h", ctypes.c_double * 3), ("bc_lo", ctypes.c_int * 3),
                ("bc_hi", ctypes.c_int * 3), ("gamma", ctypes.c_double),
                ("law", ctypes.POINTER(Law)), ("metrics", ctypes.POINTER(ctypes.c_double))]


@dataclass
class LawSpec:
    """Python view of ``sfo_law`` (values are used by fixedValue laws)."""
    rho: int = LAW_ZERO_GRADIENT
    U: int = LAW_ZERO_GRADIENT
    p: int = LAW_ZERO_GRADIENT
    rho_value: float = 0.0
    U_value: tuple = (0.0, 0.0, 0.0)
    p_value: float = 0.0

    def c(self) -> Law:
        law = Law()
        law.rho, law.U, law.p = int(self.rho), int(self.U), int(self.p)
        law.rho_value = float(self.rho_value)
        for d in range(3):
            law.U_value[d] = float(self.U_value[d])
        law.p_value = float(self.p_value)
        return law


class Counters(ctypes.Structure):
    _fields_ = [("teno_cores", ctypes.c_ulonglong), ("teno_cut", ctypes.c_ulonglong),
                ("faces", ctypes.c_ulonglong)]


@dataclass
class GridSpec:
    """Python view of ``sfo_grid``."""
    dim: int
    n: tuple
    ng: int = 3
    h: tuple = (1.0, 1.0, 1.0)
    bc_lo: tuple = (0, 0, 0)
    bc_hi: tuple = (0, 0, 0)
    gamma: float = 1.4
    laws: dict = field(default_factory=dict)   # (axis, end) -> LawSpec for BC_LAW ends
    metrics: np.ndarray | None = None          # curvilinear: (mz, my, mx, 10) over Q's layout

    def c(self) -> Grid:
        g = Grid()
        g.dim = self.dim
        for d in range(3):
            g.n[d] = int(self.n[d])
            g.h[d] = float(self.h[d])
            g.bc_lo[d] = int(self.bc_lo[d])
            g.bc_hi[d] = int(self.bc_hi[d])
        g.ng = self.ng
        g.gamma = self.gamma
        if self.laws:
            arr = (Law * 6)()
            for (axis, end), law in self.laws.items():
                arr[2 * axis + end] = law.c()
            g._laws = arr               # keeps the array alive with the struct
            g.law = ctypes.cast(arr, ctypes.POINTER(Law))
        if self.metrics is not None:
            m = np.ascontiguousarray(self.metrics, dtype=np.float64)
            assert m.shape == self.extents[::-1] + (10,), (m.shape, self.extents)
            g._metrics = m
            g.metrics = m.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        return g

    @property
    def extents(self):
        return tuple(self.n[d] + (2 * self.ng if d < self.dim else 0) for d in range(3))

    def empty(self) -> np.ndarray:
        mx, my, mz = self.extents
        return np.zeros((mz, my, mx, 5), dtype=np.float64)

    def interior(self, Q: np.ndarray) -> np.ndarray:
        """View of the node block (no ghosts) of a compact array."""
        sl = []
        for d in (2, 1, 0):
            lo = self.ng if d < self.dim else 0
            sl.append(slice(lo, lo + self.n[d]))
        return Q[tuple(sl)]


_DP = ctypes.POINTER(ctypes.c_double)


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_DP)


def _load(path):
    if not os.path.exists(path):
        return None
    return ctypes.CDLL(path)


def _sig(lib, prefix):
    G = ctypes.POINTER(Grid)
    C = ctypes.POINTER(Counters)
    # both libraries hold the restatement's step-dt slot (the reference
    # library links its own copy of sf_oracle.c)
    lib.sfo_set_step_dt.argtypes = [ctypes.c_double]
    lib.sfo_step_dt.restype = ctypes.c_double
    if prefix == "sfo":
        lib.sfo_storage_size.argtypes = [G]
        lib.sfo_storage_size.restype = ctypes.c_longlong
        for nm in ("sfo_weno3_core", "sfo_weno5_core", "sfo_weno7_core"):
            getattr(lib, nm).argtypes = [_DP]
            getattr(lib, nm).restype = ctypes.c_double
        lib.sfo_teno5_core.argtypes = [_DP, ctypes.POINTER(ctypes.c_int)]
        lib.sfo_teno5_core.restype = ctypes.c_double
        lib.sfo_char_matrix.argtypes = [_DP, _DP, ctypes.c_double, _DP, _DP]
        lib.sfo_rusanov_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfo_roe_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfo_steger_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfo_lf_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfo_lw_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, ctypes.c_double, ctypes.c_double, _DP]
        lib.sfo_char_face_flux_ex.argtypes = [ctypes.c_int, _DP, _DP, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_double, _DP]
        lib.sfo_char_face_flux.argtypes = [ctypes.c_int, _DP, _DP, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_double, _DP]
        lib.sfo_fill_ghosts.argtypes = [G, _DP]
        lib.sfo_rhs.argtypes = [G, ctypes.c_int, ctypes.c_int, _DP, _DP, C]
        lib.sfo_dt.argtypes = [G, _DP, ctypes.c_double, _DP]
        lib.sfo_step.argtypes = [G, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP, ctypes.c_double,
                                 _DP, C]
        lib.sfo_stage.argtypes = [G, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP, ctypes.c_double,
                                  ctypes.c_int, _DP, C]
        lib.sfo_advance.argtypes = [G, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_int, _DP,
                                    ctypes.POINTER(ctypes.c_int), _DP, C]
    else:
        lib.sfr_rhs.argtypes = [G, ctypes.c_int, ctypes.c_int, _DP, _DP]
        lib.sfr_fill_laws.argtypes = [G, _DP]
        lib.sfr_dt.argtypes = [G, _DP, ctypes.c_double, _DP]
        for nm in ("sfr_weno3_core", "sfr_weno5_core", "sfr_teno5_core", "sfr_weno7_core"):
            getattr(lib, nm).argtypes = [_DP]
            getattr(lib, nm).restype = ctypes.c_double
        lib.sfr_char_matrix.argtypes = [_DP, _DP, ctypes.c_double, _DP, _DP]
        lib.sfr_rusanov_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfr_roe_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfr_steger_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfr_lf_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, _DP]
        lib.sfr_lw_flux.argtypes = [_DP, _DP, _DP, ctypes.c_double, ctypes.c_double, ctypes.c_double, _DP]
        lib.sfr_case_create.argtypes = [G, ctypes.c_int, ctypes.c_int]
        lib.sfr_case_create.restype = ctypes.c_void_p
        lib.sfr_case_destroy.argtypes = [ctypes.c_void_p]
        lib.sfr_case_rhs.argtypes = [ctypes.c_void_p, _DP, _DP]
        lib.sfr_case_dt.argtypes = [ctypes.c_void_p, _DP, ctypes.c_double, _DP]
        lib.sfr_case_step.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP, ctypes.c_double]
        lib.sfr_case_advance.argtypes = [ctypes.c_void_p, ctypes.c_int, _DP, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_int, _DP,
                                         ctypes.POINTER(ctypes.c_int), _DP]
    return lib


_oracle = None
_ref = {}


def oracle_lib():
    """The C restatement (built by ``make -C oracle``)."""
    global _oracle
    if _oracle is None:
        lib = _load(os.path.join(HERE, "liboracle.so"))
        if lib is None:
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        _oracle = _sig(lib, "sfo")
    return _oracle


def host_march() -> str | None:
    """The CPU target `gcc -march=native` selects on this host (None when gcc
    cannot tell)."""
    import subprocess
    try:
        out = subprocess.run(["gcc", "-march=native", "-Q", "--help=target"], capture_output=True, text=True,
                             timeout=30).stdout
    except Exception:
        return None
    for line in out.splitlines():
        f = line.split()
        if len(f) == 2 and f[0] == "-march=":
            return f[1]
    return None


def ref_native_build() -> tuple[str, str]:
    """(library file, gcc flags) of the timed reference build for this host:
    the build for the target `gcc -march=native` selects here when oracle/_ref
    has one (the reference's own -march=native), else the x86-64-v3 build."""
    arch = host_march()
    if arch:
        name = f"libsfref_native_{arch}.so"
        if os.path.exists(os.path.join(HERE, "_ref", name)):
            return name, f"-O3 -march={arch} (gcc -march=native on this host)"
    return "libsfref_native.so", "-O3 -march=x86-64-v3"


def ref_lib(native: bool = False):
    """The reference translation units, or None when they were not built."""
    key = "native" if native else "strict"
    if key not in _ref:
        lib = _load(os.path.join(HERE, "_ref", ref_native_build()[0] if native else "libsfref.so"))
        _ref[key] = _sig(lib, "sfr") if lib is not None else None
    return _ref[key]


def _check(code, what):
    if code != 0:
        raise RuntimeError(f"{what}: {ERRORS.get(code, code)}")


class OracleError(RuntimeError):
    pass


# ---------------------------------------------------------------- restatement

def fill_ghosts(spec: GridSpec, Q: np.ndarray) -> None:
    _check(oracle_lib().sfo_fill_ghosts(ctypes.byref(spec.c()), _ptr(Q)), "fill_ghosts")


def ref_fill_laws(spec: GridSpec, Q: np.ndarray) -> None:
    """The reference's own boundary laws of the LAW ends applied to Q."""
    lib = ref_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/libsfref.so missing: run `make -C oracle`")
    _check(lib.sfr_fill_laws(ctypes.byref(spec.c()), _ptr(Q)), "ref fill_laws")


def set_step_dt(dt: float) -> None:
    """Step size the Lax-Wendroff flux sees in a bare rhs call (the stage
    and step functions set it from their own dt), in the restatement and in
    the reference library."""
    oracle_lib().sfo_set_step_dt(dt)
    ref_lib(False)
    for ref in _ref.values():
        if ref is not None:
            ref.sfo_set_step_dt(dt)


def rhs(spec: GridSpec, scheme: int, flux: int, Q: np.ndarray, counters: Counters | None = None):
    R = np.zeros_like(Q)
    code = oracle_lib().sfo_rhs(ctypes.byref(spec.c()), scheme, flux, _ptr(Q), _ptr(R),
                                ctypes.byref(counters) if counters is not None else None)
    _check(code, "rhs")
    return R


def dt(spec: GridSpec, Q: np.ndarray, cfl: float) -> float:
    out = ctypes.c_double()
    _check(oracle_lib().sfo_dt(ctypes.byref(spec.c()), _ptr(Q), cfl, ctypes.byref(out)), "dt")
    return out.value


class Stepper:
    """Holds the q0 / k work arrays between stages of one step."""

    def __init__(self, spec: GridSpec, scheme: int, flux: int, time_id: int):
        self.spec, self.scheme, self.flux, self.time_id = spec, scheme, flux, time_id
        self.g = spec.c()
        self.work = np.zeros(5 * int(oracle_lib().sfo_storage_size(ctypes.byref(self.g))))
        self.counters = Counters()

    def stage(self, Q, dt_, s):
        code = oracle_lib().sfo_stage(ctypes.byref(self.g), self.scheme, self.flux, self.time_id,
                                      _ptr(Q), dt_, s, _ptr(self.work), ctypes.byref(self.counters))
        if code:
            raise OracleError(f"stage {s}: {ERRORS.get(code, code)}")

    def step(self, Q, dt_):
        code = oracle_lib().sfo_step(ctypes.byref(self.g), self.scheme, self.flux, self.time_id,
                                     _ptr(Q), dt_, _ptr(self.work), ctypes.byref(self.counters))
        if code:
            raise OracleError(f"step: {ERRORS.get(code, code)}")


def advance(spec: GridSpec, scheme, flux, time_id, Q, t_end, cfl, *, t_start=0.0,
            max_dt=1.7976931348623157e308, write_interval=0.0, max_steps=10 ** 7,
            counters: Counters | None = None):
    """Runs the Time::Driver loop; returns (dt array, t_final)."""
    cap = min(max_steps, 10 ** 7)
    dts = np.zeros(cap)
    steps = ctypes.c_int()
    tf = ctypes.c_double()
    code = oracle_lib().sfo_advance(ctypes.byref(spec.c()), scheme, flux, time_id, _ptr(Q),
                                    t_start, t_end, cfl, max_dt, write_interval, cap, _ptr(dts),
                                    ctypes.byref(steps), ctypes.byref(tf),
                                    ctypes.byref(counters) if counters is not None else None)
    if code:
        raise OracleError(f"advance: {ERRORS.get(code, code)} after {steps.value} steps")
    return dts[:steps.value].copy(), tf.value


# ---------------------------------------------------------------- reference TUs

class RefCase:
    """A persistent reference Field driven through the reference operator."""

    def __init__(self, spec: GridSpec, scheme: int, flux: int, native: bool = False):
        lib = ref_lib(native)
        if lib is None:
            raise RuntimeError("oracle/_ref not built (reference sources unavailable)")
        self.lib = lib
        self.spec = spec
        self.g = spec.c()
        self.h = lib.sfr_case_create(ctypes.byref(self.g), scheme, flux)
        if not self.h:
            raise RuntimeError("sfr_case_create failed")

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.sfr_case_destroy(self.h)
            self.h = None

    def rhs(self, Q):
        R = np.zeros_like(Q)
        _check(self.lib.sfr_case_rhs(self.h, _ptr(Q), _ptr(R)), "ref rhs")
        return R

    def dt(self, Q, cfl):
        out = ctypes.c_double()
        _check(self.lib.sfr_case_dt(self.h, _ptr(Q), cfl, ctypes.byref(out)), "ref dt")
        return out.value

    def step(self, time_id, Q, dt_):
        _check(self.lib.sfr_case_step(self.h, time_id, _ptr(Q), dt_), "ref step")

    def advance(self, time_id, Q, t_end, cfl, *, t_start=0.0, max_dt=1.7976931348623157e308,
                write_interval=0.0, max_steps=10 ** 7):
        cap = min(max_steps, 10 ** 7)
        dts = np.zeros(cap)
        steps = ctypes.c_int()
        tf = ctypes.c_double()
        code = self.lib.sfr_case_advance(self.h, time_id, _ptr(Q), t_start, t_end, cfl, max_dt,
                                         write_interval, cap, _ptr(dts), ctypes.byref(steps),
                                         ctypes.byref(tf))
        _check(code, "ref advance")
        return dts[:steps.value].copy(), tf.value


# ------------------------------------------------------------ block geometry

_mesh = None


def ref_mesh_lib():
    """The reference's structured-block generator (oracle/_ref/libsfmesh.so),
    or None when it was not built."""
    global _mesh
    if _mesh is None:
        lib = _load(os.path.join(HERE, "_ref", "libsfmesh.so"))
        if lib is None:
            return None
        IP = ctypes.POINTER(ctypes.c_int)
        lib.sfr_mesh_points.argtypes = [ctypes.c_int, _DP, ctypes.c_double, IP, IP, _DP, ctypes.c_int, IP, _DP, _DP]
        lib.sfr_mesh_points.restype = ctypes.c_int
        _mesh = lib
    return _mesh


def ref_mesh_points(vertices, hex, cells, grading=(1.0, 1.0, 1.0), edges=(), scale=1.0):
    """Node coordinates of one block from the reference's own generator
    (MeshGen::generateStructuredMesh, SF_meshGen.cpp:76-110): trilinear with
    grading, or transfinite interpolation when `edges` ((v0, v1, point) arcs)
    are given.  Returns (nz, ny, nx, 3)."""
    lib = ref_mesh_lib()
    if lib is None:
        raise RuntimeError("oracle/_ref/libsfmesh.so missing: run `make -C oracle`")
    V = np.ascontiguousarray(vertices, dtype=np.float64).reshape(-1, 3)
    H = np.ascontiguousarray(hex, dtype=np.int32)
    C = np.ascontiguousarray(cells, dtype=np.int32)
    G = np.ascontiguousarray(grading, dtype=np.float64)
    E = np.ascontiguousarray([[a, b] for a, b, _ in edges] or [[0, 0]], dtype=np.int32)
    P = np.ascontiguousarray([p for _, _, p in edges] or [[0.0, 0.0, 0.0]], dtype=np.float64)
    out = np.zeros((C[2] + 1, C[1] + 1, C[0] + 1, 3))
    IP = ctypes.POINTER(ctypes.c_int)
    code = lib.sfr_mesh_points(len(V), _ptr(V), float(scale), H.ctypes.data_as(IP), C.ctypes.data_as(IP), _ptr(G),
                               len(edges), E.ctypes.data_as(IP), _ptr(P), _ptr(out))
    _check(code, "ref mesh points")
    return out


def field_metrics(points: np.ndarray, ng: int, active=(True, True, True)):
    """The reference Field's metrics of a block (numpy restatement): ghost
    coordinates extrapolated linearly along x, then y, then z
    (Mesh::generateGhostCells, src/infrastructure/mesh/SF_mesh.cpp:491-533);
    symmetric conservative cofactors and J = (r_xi.c_xi + r_eta.c_eta +
    r_zeta.c_zeta) / 3 on every point one layer in, Jac = 1 / J and the
    metric rows = cofactors * Jac (Mesh::computeMetrics, :219-345); the
    outermost layer copied from its inner neighbour along x, then y, then z
    (applyBoundaryMetrics, :439-474).  Returns (metrics (MZ, MY, MX, 10) with
    ng ghost layers on every axis, identity residual, identity tolerance)
    with the audit of Mesh::auditMetricIdentity (:348-437) over the nodes and
    the active axes.  `points`: (nz, ny, nx, 3) node coordinates."""
    nz, ny, nx, _ = points.shape
    X = np.zeros((nz + 2 * ng, ny + 2 * ng, nx + 2 * ng, 3))
    X[ng:ng + nz, ng:ng + ny, ng:ng + nx] = points
    for ax in (2, 1, 0):                       # numpy axis of x, y, z
        M = X.shape[ax]

        def sl(i):
            s = [slice(None)] * 4
            s[ax] = i
            return tuple(s)
        for i in range(ng - 1, -1, -1):
            X[sl(i)] = 2.0 * X[sl(i + 1)] - X[sl(i + 2)]
        for i in range(M - ng, M):
            X[sl(i)] = 2.0 * X[sl(i - 1)] - X[sl(i - 2)]
    npax = {0: 2, 1: 1, 2: 0}                  # coordinate axis -> numpy axis

    def shift(A, a, o):
        return np.roll(A, -o, axis=npax[a])

    def dco(A, a):                             # central difference along axis a (valid away from its ends)
        return 0.5 * (shift(A, a, 1) - shift(A, a, -1))

    D = {(c, a): dco(X[..., c], a) for c in range(3) for a in range(3)}

    def dprod(p, q, inner, outer):
        P = X[..., p] * D[(q, inner)]
        return 0.5 * (shift(P, outer, 1) - shift(P, outer, -1))

    after1, after2 = (1, 2, 0), (2, 0, 1)
    cof = {}
    for a_ in range(3):
        a, b = after1[a_], after2[a_]
        for c in range(3):
            p, q = after1[c], after2[c]
            curl1 = dprod(p, q, b, a) - dprod(p, q, a, b)
            curl2 = dprod(q, p, a, b) - dprod(q, p, b, a)
            cof[(a_, c)] = 0.5 * (curl1 + curl2)

    def rowdot(a):
        return D[(0, a)] * cof[(a, 0)] + D[(1, a)] * cof[(a, 1)] + D[(2, a)] * cof[(a, 2)]
    J = (rowdot(0) + rowdot(1) + rowdot(2)) / 3.0
    inner = (slice(1, -1),) * 3
    Mt = np.zeros(X.shape[:3] + (10,))
    Jac = 1.0 / J[inner]
    Mt[inner + (0,)] = Jac
    for a in range(3):
        for c in range(3):
            Mt[inner + (1 + 3 * a + c,)] = cof[(a, c)][inner] * Jac
    Mt[:, :, 0] = Mt[:, :, 1]
    Mt[:, :, -1] = Mt[:, :, -2]
    Mt[:, 0] = Mt[:, 1]
    Mt[:, -1] = Mt[:, -2]
    Mt[0] = Mt[1]
    Mt[-1] = Mt[-2]
    nodes = (slice(ng, ng + nz), slice(ng, ng + ny), slice(ng, ng + nx))
    div = np.zeros((nz, ny, nx, 3))
    cmax = 0.0
    for a in range(3):
        if not active[a]:
            continue
        F = 0.5 * (Mt[..., 1 + 3 * a:4 + 3 * a] / Mt[..., :1] +
                   shift(Mt[..., 1 + 3 * a:4 + 3 * a] / Mt[..., :1], a, 1))
        fp, fm = F[nodes], shift(F, a, -1)[nodes]
        cmax = max(cmax, float(np.abs(fp).max()), float(np.abs(fm).max()))
        div = div + (fp - fm)
    tol = 65536.0 * np.finfo(float).eps * max(cmax, np.finfo(float).tiny)
    return Mt, float(np.abs(div).max()), tol
