"""ctypes binding of the C ABI in ``include/sonicsolver_b200.h``.

This is the Python face of the B200 provider: it loads the in-tree
``libsonicsolver_b200.so`` (built by :mod:`sonicsolver_b200.build`) and raises
if it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsonicsolver_b200.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_STATE, ERR_TENO_CUTOFF, ERR_NOMEM, ERR_BUDGET, ERR_TIMEOUT, ERR_NOT_FOUND, ERR_CANCELLED = range(1, 10)

FLAG_NONFINITE, FLAG_DENSITY, FLAG_PRESSURE, FLAG_TENO_CUTOFF, FLAG_ROE_SOUND = 1, 2, 4, 8, 16

# FDM::TermRecipeId values: scheme * 5 + face flux (Steger, Rusanov,
# LaxFriedrichs, Roe, LaxWendroff).
RECIPES = {f"{sch}{flx}": 5 * i + j
           for i, sch in enumerate(("weno3", "weno5", "teno5", "weno7"))
           for j, flx in enumerate(("Steger", "Rusanov", "LaxFriedrichs", "Roe", "LaxWendroff"))}
TIME_RECIPES = {"forwardEuler": 0, "SSPRK3": 1, "classicalRK4": 2}
PREC_FP64, PREC_FP32_FLUX = 0, 1
BC_TRANSMISSIVE, BC_PERIODIC, BC_FROZEN, BC_LAW = 0, 1, 2, 3
LAW_ZERO_GRADIENT, LAW_FIXED_VALUE, LAW_SYMMETRY = 0, 1, 2
LAYOUT_NODES, LAYOUT_FIELD = 0, 1

# The C-ABI symbols declared by include/sonicsolver_b200.h (checked by tests).
EXPORTS = (
    "sfg_last_error", "sfg_version", "sfg_recipe_name", "sfg_recipe_from_name", "sfg_create",
    "sfg_destroy", "sfg_ghost_layers", "sfg_state_size", "sfg_upload", "sfg_restore", "sfg_download",
    "sfg_upload_device", "sfg_download_device", "sfg_compute_dt", "sfg_stage", "sfg_step",
    "sfg_advance", "sfg_residual", "sfg_stage_with_residual", "sfg_conserved_totals", "sfg_time",
    "sfg_status_word", "sfg_set_counting", "sfg_get_counters", "sfg_time_sweeps", "sfg_measure_fma_peak",
)


class GridDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n", ctypes.c_int * 3), ("h", ctypes.c_double * 3),
                ("bc_lo", ctypes.c_int * 3), ("bc_hi", ctypes.c_int * 3)]


class BoundaryLaw(ctypes.Structure):
    """``sfg_boundary_law``: density / velocity / pressure law of one law end."""
    _fields_ = [("rho", ctypes.c_int), ("velocity", ctypes.c_int), ("pressure", ctypes.c_int),
                ("reserved", ctypes.c_int), ("rho_value", ctypes.c_double),
                ("velocity_value", ctypes.c_double * 3), ("pressure_value", ctypes.c_double)]


def law_array(laws):
    """The laws of a grid's law ends as the C ABI takes them
    (laws[2 * axis + end]) from {(axis, end): dict(rho=, velocity=, pressure=,
    rho_value=, velocity_value=, pressure_value=)}; None when `laws` is
    empty."""
    if not laws:
        return None
    arr = (BoundaryLaw * 6)()
    for (axis, end), kw in laws.items():
        law = arr[2 * axis + end]
        law.rho = int(kw.get("rho", LAW_ZERO_GRADIENT))
        law.velocity = int(kw.get("velocity", LAW_ZERO_GRADIENT))
        law.pressure = int(kw.get("pressure", LAW_ZERO_GRADIENT))
        law.rho_value = float(kw.get("rho_value", 0.0))
        for d, v in enumerate(kw.get("velocity_value", (0.0, 0.0, 0.0))):
            law.velocity_value[d] = float(v)
        law.pressure_value = float(kw.get("pressure_value", 0.0))
    return arr


class NumericsDesc(ctypes.Structure):
    _fields_ = [("recipe", ctypes.c_int), ("time_recipe", ctypes.c_int), ("precision", ctypes.c_int),
                ("gamma", ctypes.c_double), ("cfl", ctypes.c_double), ("max_dt", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("steps", ctypes.c_int64), ("time", ctypes.c_double), ("last_dt", ctypes.c_double),
                ("device_ms", ctypes.c_double), ("status_bits", ctypes.c_uint32),
                ("teno_cut", ctypes.c_uint64), ("teno_cores", ctypes.c_uint64)]


class RequestInfo(ctypes.Structure):
    _fields_ = [("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("finish_s", ctypes.c_double),
                ("steps", ctypes.c_int64), ("time", ctypes.c_double), ("flags", ctypes.c_uint32),
                ("state", ctypes.c_int)]


REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = range(5)


class SolverError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_DP = ctypes.POINTER(ctypes.c_double)
_VP = ctypes.c_void_p


def lib():
    """The loaded provider library (raises when it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m sonicsolver_b200.build` "
                               "(the provider has no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        L.sfg_last_error.restype = ctypes.c_char_p
        L.sfg_recipe_name.restype = ctypes.c_char_p
        L.sfg_recipe_name.argtypes = [ctypes.c_int]
        L.sfg_recipe_from_name.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]
        L.sfg_version.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.sfg_create.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(NumericsDesc), _VP, ctypes.POINTER(_VP)]
        L.sfg_destroy.argtypes = [_VP]
        L.sfg_ghost_layers.argtypes = [_VP, ctypes.POINTER(ctypes.c_int)]
        L.sfg_set_boundary_law.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(BoundaryLaw)]
        L.sfg_apply_boundary.argtypes = [_VP]
        L.sfg_set_metrics.argtypes = [_VP, _DP, ctypes.c_int]
        L.sfg_state_size.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
        L.sfg_upload.argtypes = [_VP, _DP, ctypes.c_int, ctypes.c_double]
        L.sfg_restore.argtypes = [_VP, _DP, ctypes.c_int, ctypes.c_double, ctypes.c_int64]
        L.sfg_download.argtypes = [_VP, _DP, ctypes.c_int]
        L.sfg_upload_device.argtypes = [_VP, _VP, ctypes.c_double]
        L.sfg_download_device.argtypes = [_VP, _VP]
        L.sfg_compute_dt.argtypes = [_VP, ctypes.c_double, _DP]
        L.sfg_stage.argtypes = [_VP, ctypes.c_int, ctypes.c_double]
        L.sfg_step.argtypes = [_VP, ctypes.c_double, ctypes.c_double]
        L.sfg_advance.argtypes = [_VP, ctypes.c_double, ctypes.c_int64, ctypes.c_double, ctypes.c_int, _DP,
                                  ctypes.c_int64, ctypes.POINTER(Stats)]
        L.sfg_residual.argtypes = [_VP, _DP]
        L.sfg_stage_with_residual.argtypes = [_VP, ctypes.c_int, ctypes.c_double, _DP]
        L.sfg_conserved_totals.argtypes = [_VP, _DP]
        L.sfg_time.argtypes = [_VP, _DP, ctypes.POINTER(ctypes.c_int64)]
        L.sfg_status_word.argtypes = [_VP, ctypes.POINTER(ctypes.c_uint32), ctypes.c_int]
        L.sfg_set_counting.argtypes = [_VP, ctypes.c_int]
        L.sfg_get_counters.argtypes = [_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.sfg_time_sweeps.argtypes = [_VP, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_float)]
        L.sfg_measure_fma_peak.argtypes = [ctypes.c_int, ctypes.c_double, _DP]
        L.sfg_residual_noalloc.argtypes = [ctypes.POINTER(GridDesc), ctypes.POINTER(NumericsDesc), _VP, _VP, _VP]
        L.sfg_set_kernel_variant.argtypes = [_VP, ctypes.c_int]
        L.sfg_get_kernel_variant.argtypes = [_VP, ctypes.POINTER(ctypes.c_int)]
        L.sfg_teno_flip_rate.argtypes = [_VP, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        PG, PN = ctypes.POINTER(GridDesc), ctypes.POINTER(NumericsDesc)
        I64P = ctypes.POINTER(ctypes.c_int64)
        L.sfg_batch_create.argtypes = [PN, ctypes.c_size_t, ctypes.c_int, _VP, ctypes.POINTER(_VP)]
        L.sfg_batch_destroy.argtypes = [_VP]
        L.sfg_batch_instance_bytes.argtypes = [_VP, PG, ctypes.POINTER(ctypes.c_size_t)]
        L.sfg_batch_add.argtypes = [_VP, PG, _DP, ctypes.c_double, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]
        L.sfg_batch_add_ex.argtypes = [_VP, PG, PN, _DP, ctypes.c_double, ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]
        PL = ctypes.POINTER(BoundaryLaw)
        L.sfg_batch_add_laws.argtypes = [_VP, PG, PN, PL, _DP, ctypes.c_double, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int)]
        L.sfg_batch_remove.argtypes = [_VP, ctypes.c_int]
        L.sfg_batch_set_write_interval.argtypes = [_VP, ctypes.c_int, ctypes.c_double]
        L.sfg_batch_step.argtypes = [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.sfg_batch_status.argtypes = [_VP, ctypes.c_int, _DP, I64P, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_uint32)]
        L.sfg_batch_download.argtypes = [_VP, ctypes.c_int, _DP]
        L.sfg_batch_set_variant.argtypes = [_VP, ctypes.c_int]
        L.sfg_batch_info.argtypes = [_VP, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.sfg_batch_snapshot.argtypes = [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP, I64P,
                                         ctypes.POINTER(ctypes.c_uint32)]
        L.sfg_server_create.argtypes = [PN, ctypes.c_size_t, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP)]
        L.sfg_server_destroy.argtypes = [_VP]
        L.sfg_server_submit.argtypes = [_VP, PG, _DP, ctypes.c_double, ctypes.c_int64, I64P]
        L.sfg_server_submit_ex.argtypes = [_VP, PG, PN, _DP, ctypes.c_double, ctypes.c_int64, I64P]
        L.sfg_server_submit_laws.argtypes = [_VP, PG, PN, ctypes.POINTER(BoundaryLaw), _DP, ctypes.c_double,
                                             ctypes.c_int64, I64P]
        L.sfg_server_poll.argtypes = [_VP, ctypes.c_int64, ctypes.POINTER(RequestInfo)]
        L.sfg_server_fetch.argtypes = [_VP, ctypes.c_int64, _DP]
        L.sfg_server_cancel.argtypes = [_VP, ctypes.c_int64]
        L.sfg_server_drain.argtypes = [_VP, ctypes.c_double]
        L.sfg_server_now.argtypes = [_VP]
        L.sfg_server_now.restype = ctypes.c_double
        _lib = L
    return _lib


def check(code: int):
    if code != OK:
        raise SolverError(code, lib().sfg_last_error().decode())


def _dptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("expected a C-contiguous float64 array")
    return a.ctypes.data_as(_DP)


def grid_desc(dim, n, h, bc_lo, bc_hi) -> GridDesc:
    g = GridDesc()
    g.dim = dim
    for d in range(3):
        g.n[d] = int(n[d])
        g.h[d] = float(h[d])
        g.bc_lo[d] = int(bc_lo[d])
        g.bc_hi[d] = int(bc_hi[d])
    return g


class Solver:
    """One grid on the GPU (``sfg_solver``)."""

    def __init__(self, dim, n, h, bc_lo, bc_hi, recipe="weno5Rusanov", time_recipe="SSPRK3",
                 precision=PREC_FP64, gamma=1.4, cfl=0.5, max_dt=0.0, stream=None):
        self.dim, self.n = dim, tuple(int(x) for x in n)
        g = grid_desc(dim, n, h, bc_lo, bc_hi)
        nm = NumericsDesc()
        nm.recipe = RECIPES[recipe] if isinstance(recipe, str) else int(recipe)
        nm.time_recipe = TIME_RECIPES[time_recipe] if isinstance(time_recipe, str) else int(time_recipe)
        nm.precision = precision
        nm.gamma, nm.cfl, nm.max_dt = gamma, cfl, max_dt
        h_ = _VP()
        check(lib().sfg_create(ctypes.byref(g), ctypes.byref(nm), stream, ctypes.byref(h_)))
        self._h = h_

    def close(self):
        if getattr(self, "_h", None):
            lib().sfg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def node_shape(self):
        return (self.n[2], self.n[1], self.n[0], 5)

    def set_boundary_law(self, axis, end, rho=LAW_ZERO_GRADIENT, velocity=LAW_ZERO_GRADIENT,
                         pressure=LAW_ZERO_GRADIENT, rho_value=0.0, velocity_value=(0.0, 0.0, 0.0),
                         pressure_value=0.0):
        """Laws of a BC_LAW end (axis, end 0 = low / 1 = high)."""
        law = BoundaryLaw()
        law.rho, law.velocity, law.pressure = int(rho), int(velocity), int(pressure)
        law.rho_value = float(rho_value)
        for d in range(3):
            law.velocity_value[d] = float(velocity_value[d])
        law.pressure_value = float(pressure_value)
        check(lib().sfg_set_boundary_law(self._h, axis, end, ctypes.byref(law)))

    def set_metrics(self, metrics: np.ndarray, layout=LAYOUT_NODES):
        """Per-node metrics (Jac, xi_x..zeta_z: 10 per node) of a curvilinear grid."""
        m = np.ascontiguousarray(metrics, dtype=np.float64)
        check(lib().sfg_set_metrics(self._h, _dptr(m), layout))

    def apply_boundary(self):
        """Apply the laws of every law end to the current state once."""
        check(lib().sfg_apply_boundary(self._h))

    def upload(self, q: np.ndarray, time: float = 0.0, layout=LAYOUT_NODES):
        check(lib().sfg_upload(self._h, _dptr(q), layout, time))

    def restore(self, q: np.ndarray, time: float, steps: int, layout=LAYOUT_NODES):
        """Resume a run: the state, its time and its step count (as `time()`
        reported them when the state was downloaded)."""
        check(lib().sfg_restore(self._h, _dptr(q), layout, time, int(steps)))

    def download(self, layout=LAYOUT_NODES, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            cnt = ctypes.c_size_t()
            check(lib().sfg_state_size(self._h, layout, ctypes.byref(cnt)))
            out = np.empty(cnt.value, dtype=np.float64)
        check(lib().sfg_download(self._h, _dptr(out), layout))
        return out

    def compute_dt(self, limit=0.0) -> float:
        v = ctypes.c_double()
        check(lib().sfg_compute_dt(self._h, limit, ctypes.byref(v)))
        return v.value

    def stage(self, s, dt):
        check(lib().sfg_stage(self._h, s, dt))

    def step(self, dt=0.0, limit=0.0):
        check(lib().sfg_step(self._h, dt, limit))

    def advance(self, t_end, max_steps=0, write_interval=0.0, graph_steps=0, dt_capacity=0):
        st = Stats()
        buf = np.zeros(max(dt_capacity, 1))
        check(lib().sfg_advance(self._h, t_end, max_steps, write_interval, graph_steps,
                                _dptr(buf) if dt_capacity else None, dt_capacity, ctypes.byref(st)))
        return st, buf[:min(st.steps, dt_capacity)].copy() if dt_capacity else None

    def residual(self) -> np.ndarray:
        out = np.empty(5 * int(np.prod(self.n)), dtype=np.float64)
        check(lib().sfg_residual(self._h, _dptr(out)))
        return out

    def stage_with_residual(self, s, dt, r: np.ndarray):
        check(lib().sfg_stage_with_residual(self._h, s, dt, _dptr(np.ascontiguousarray(r, dtype=np.float64))))

    def totals(self):
        out = np.zeros(5)
        check(lib().sfg_conserved_totals(self._h, _dptr(out)))
        return out

    def time(self):
        t = ctypes.c_double()
        n = ctypes.c_int64()
        check(lib().sfg_time(self._h, ctypes.byref(t), ctypes.byref(n)))
        return t.value, n.value

    def status(self, clear=False):
        b = ctypes.c_uint32()
        check(lib().sfg_status_word(self._h, ctypes.byref(b), 1 if clear else 0))
        return b.value

    def set_counting(self, on=True):
        check(lib().sfg_set_counting(self._h, 1 if on else 0))

    def counters(self):
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().sfg_get_counters(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    @property
    def variant(self) -> int:
        v = ctypes.c_int()
        check(lib().sfg_get_kernel_variant(self._h, ctypes.byref(v)))
        return v.value

    @variant.setter
    def variant(self, v: int):
        check(lib().sfg_set_kernel_variant(self._h, int(v)))

    def teno_flips(self):
        """(decisions, flips) of TENO5 cut-offs, FP64 vs FP32 on the current state."""
        d, f = ctypes.c_uint64(), ctypes.c_uint64()
        check(lib().sfg_teno_flip_rate(self._h, ctypes.byref(d), ctypes.byref(f)))
        return d.value, f.value

    def time_sweeps(self, dt, stage=0, repeats=5):
        out = (ctypes.c_float * 3)()
        check(lib().sfg_time_sweeps(self._h, stage, dt, repeats, out))
        return [out[d] for d in range(self.dim)]


def numerics_desc(recipe="weno5Rusanov", time_recipe="SSPRK3", precision=PREC_FP64, gamma=1.4, cfl=0.5,
                  max_dt=0.0) -> NumericsDesc:
    nm = NumericsDesc()
    nm.recipe = RECIPES[recipe] if isinstance(recipe, str) else int(recipe)
    nm.time_recipe = TIME_RECIPES[time_recipe] if isinstance(time_recipe, str) else int(time_recipe)
    nm.precision = precision
    nm.gamma, nm.cfl, nm.max_dt = gamma, cfl, max_dt
    return nm


def _own_numerics(defaults: dict, recipe, gamma, cfl, max_dt):
    """A grid's own numerics (sfg_batch_add_ex / sfg_server_submit_ex): the
    given fields over the batch's or server's, or None when none is given."""
    if recipe is None and gamma is None and cfl is None and max_dt is None:
        return None
    d = dict(defaults)
    for k, v in (("recipe", recipe), ("gamma", gamma), ("cfl", cfl), ("max_dt", max_dt)):
        if v is not None:
            d[k] = v
    return numerics_desc(**d)


class Batch:
    """Many independent 1-D / 2-D grids stepped together (sfg_batch).  A grid
    added with its own recipe / gamma / CFL / maxDeltaT runs with them."""

    def __init__(self, budget_bytes, max_instances, recipe="weno5Rusanov", time_recipe="SSPRK3",
                 precision=PREC_FP64, gamma=1.4, cfl=0.5, max_dt=0.0, stream=None):
        self.defaults = dict(recipe=recipe, time_recipe=time_recipe, precision=precision, gamma=gamma, cfl=cfl,
                             max_dt=max_dt)
        nm = numerics_desc(recipe, time_recipe, precision, gamma, cfl, max_dt)
        h = _VP()
        check(lib().sfg_batch_create(ctypes.byref(nm), int(budget_bytes), int(max_instances), stream, ctypes.byref(h)))
        self._h = h
        self.shapes = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().sfg_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add(self, case, t_end=None, max_steps=0, recipe=None, gamma=None, cfl=None, max_dt=None, laws=None) -> int:
        """A grid with its own numerics where given; `laws` ({(axis, end):
        dict}, see law_array) for its BC_LAW ends."""
        g = grid_desc(case.dim, case.n, case.h, case.bc_lo, case.bc_hi)
        slot = ctypes.c_int()
        q = np.ascontiguousarray(case.q, dtype=np.float64)
        nm = _own_numerics(self.defaults, recipe, gamma, cfl, max_dt)
        check(lib().sfg_batch_add_laws(self._h, ctypes.byref(g), ctypes.byref(nm) if nm is not None else None,
                                       law_array(laws), _dptr(q), case.t_end if t_end is None else t_end, max_steps,
                                       ctypes.byref(slot)))
        self.shapes[slot.value] = q.shape
        return slot.value

    def instance_bytes(self, case) -> int:
        g = grid_desc(case.dim, case.n, case.h, case.bc_lo, case.bc_hi)
        b = ctypes.c_size_t()
        check(lib().sfg_batch_instance_bytes(self._h, ctypes.byref(g), ctypes.byref(b)))
        return b.value

    def set_write_interval(self, slot, write_interval):
        """Clip the grid's steps at every write_interval (as sfg_advance)."""
        check(lib().sfg_batch_set_write_interval(self._h, slot, float(write_interval)))

    def remove(self, slot):
        check(lib().sfg_batch_remove(self._h, slot))
        self.shapes.pop(slot, None)

    def step(self, steps, graph_steps=16) -> int:
        a = ctypes.c_int()
        check(lib().sfg_batch_step(self._h, int(steps), int(graph_steps), ctypes.byref(a)))
        return a.value

    def status(self, slot):
        t, n, r, f = ctypes.c_double(), ctypes.c_int64(), ctypes.c_int(), ctypes.c_uint32()
        check(lib().sfg_batch_status(self._h, slot, ctypes.byref(t), ctypes.byref(n), ctypes.byref(r), ctypes.byref(f)))
        return {"time": t.value, "steps": n.value, "running": bool(r.value), "flags": f.value}

    def download(self, slot) -> np.ndarray:
        out = np.empty(self.shapes[slot], dtype=np.float64)
        check(lib().sfg_batch_download(self._h, slot, _dptr(out)))
        return out

    @property
    def variant(self):
        raise AttributeError("write-only")

    @variant.setter
    def variant(self, v):
        check(lib().sfg_batch_set_variant(self._h, int(v)))

    def info(self):
        u, b, l, i = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_int(), ctypes.c_int()
        check(lib().sfg_batch_info(self._h, ctypes.byref(u), ctypes.byref(b), ctypes.byref(l), ctypes.byref(i)))
        return {"used": u.value, "budget": b.value, "live": l.value, "items": i.value}


class Server:
    """Continuous-batching request loop (sfg_server) on its own host thread.
    A request submitted with its own recipe / gamma / CFL / maxDeltaT runs
    with them."""

    def __init__(self, budget_bytes, max_slots, recipe="weno5Rusanov", time_recipe="SSPRK3", precision=PREC_FP64,
                 gamma=1.4, cfl=0.5, graph_steps=16):
        self.defaults = dict(recipe=recipe, time_recipe=time_recipe, precision=precision, gamma=gamma, cfl=cfl,
                             max_dt=0.0)
        nm = numerics_desc(recipe, time_recipe, precision, gamma, cfl)
        h = _VP()
        check(lib().sfg_server_create(ctypes.byref(nm), int(budget_bytes), int(max_slots), int(graph_steps),
                                      ctypes.byref(h)))
        self._h = h
        self.shapes = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().sfg_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, case, t_end=None, max_steps=0, recipe=None, gamma=None, cfl=None, max_dt=None,
               laws=None) -> int:
        g = grid_desc(case.dim, case.n, case.h, case.bc_lo, case.bc_hi)
        q = np.ascontiguousarray(case.q, dtype=np.float64)
        rid = ctypes.c_int64()
        nm = _own_numerics(self.defaults, recipe, gamma, cfl, max_dt)
        check(lib().sfg_server_submit_laws(self._h, ctypes.byref(g), ctypes.byref(nm) if nm is not None else None,
                                           law_array(laws), _dptr(q), case.t_end if t_end is None else t_end,
                                           int(max_steps), ctypes.byref(rid)))
        self.shapes[rid.value] = q.shape
        return rid.value

    def poll(self, rid) -> RequestInfo:
        info = RequestInfo()
        check(lib().sfg_server_poll(self._h, rid, ctypes.byref(info)))
        return info

    def fetch(self, rid) -> np.ndarray:
        out = np.empty(self.shapes[rid], dtype=np.float64)
        check(lib().sfg_server_fetch(self._h, rid, _dptr(out)))
        return out

    def cancel(self, rid):
        check(lib().sfg_server_cancel(self._h, rid))

    def drain(self, timeout_s=600.0):
        check(lib().sfg_server_drain(self._h, float(timeout_s)))

    def now(self) -> float:
        return lib().sfg_server_now(self._h)


NOALLOC_MAX_NODES = 262144  # SFG_NOALLOC_MAX_NODES in include/sonicsolver_b200.h


def residual_noalloc(dim, n, h, bc_lo, bc_hi, dev_q: int, dev_r: int, recipe="weno5Rusanov",
                     precision=PREC_FP64, gamma=1.4, stream=None):
    """sfg_residual_noalloc on caller-owned device arrays (addresses as ints,
    structure of arrays [5][nodes]).  For callers that cannot allocate device
    memory themselves at this point; the library allocates nothing either."""
    g = grid_desc(dim, n, h, bc_lo, bc_hi)
    nm = NumericsDesc()
    nm.recipe = RECIPES[recipe] if isinstance(recipe, str) else int(recipe)
    nm.time_recipe = TIME_RECIPES["SSPRK3"]
    nm.precision = precision
    nm.gamma, nm.cfl, nm.max_dt = gamma, 0.5, 0.0
    check(lib().sfg_residual_noalloc(ctypes.byref(g), ctypes.byref(nm), _VP(dev_q), _VP(dev_r), stream))


def fma_peak_tflops(fp64=True, seconds=0.5) -> float:
    v = ctypes.c_double()
    check(lib().sfg_measure_fma_peak(1 if fp64 else 0, seconds, ctypes.byref(v)))
    return v.value
