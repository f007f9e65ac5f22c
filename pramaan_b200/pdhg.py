"""Host-side mirror of the reference's GPU PDHG interface.

Same names, argument meaning and error behaviour as the reference's C++ API
(include/pramaan/gpu/pdhg_solver.hpp, include/pramaan/simplex.hpp,
include/pramaan/ir.hpp and the test-harness launchers of src/gpu/pdhg.cu),
implemented over the C ABI of libpramaan_b200.so.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L

kInfinity = 1.0e30   # include/pramaan/ir.hpp:47

# PdhgOptions.algorithm / .termination values (include/pramaan_b200.h)
ALGO_REFERENCE, ALGO_ADAPTIVE, ALGO_HALPERN = 0, 1, 2
TERM_REFERENCE, TERM_RELATIVE_KKT = 0, 1


class ObjSense(enum.IntEnum):
    kMinimize = 0
    kMaximize = 1


class SolveStatus(enum.IntEnum):
    """include/pramaan/simplex.hpp:26-33"""
    kOptimal = 0
    kInfeasible = 1
    kUnbounded = 2
    kIterationLimit = 3
    kNumericalFailure = 4
    kWarmStartRejected = 5


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _ptr(a: np.ndarray | None):
    return None if a is None or a.size == 0 else a.ctypes.data_as(C.c_void_p)


@dataclass
class ModelIR:
    """LP in the reference's ranged form (include/pramaan/ir.hpp:62-119):
    optimize obj_sense c^T x + obj_offset s.t. row_lower <= A x <= row_upper,
    var_lower <= x <= var_upper, A in CSR with int32 indices."""
    obj_coeffs: np.ndarray
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    var_lower: np.ndarray
    var_upper: np.ndarray
    obj_sense: ObjSense = ObjSense.kMinimize
    obj_offset: float = 0.0

    def __post_init__(self):
        self.obj_coeffs = _f64(self.obj_coeffs)
        self.row_ptr = _i32(self.row_ptr if len(self.row_ptr) else [0])
        self.col_idx = _i32(self.col_idx)
        self.values = _f64(self.values)
        self.row_lower = _f64(self.row_lower)
        self.row_upper = _f64(self.row_upper)
        self.var_lower = _f64(self.var_lower)
        self.var_upper = _f64(self.var_upper)
        self.obj_sense = ObjSense(int(self.obj_sense))
        n, m = len(self.obj_coeffs), len(self.row_ptr) - 1
        if len(self.var_lower) != n or len(self.var_upper) != n:
            raise ValueError("ModelIR: var bounds size != num_vars")
        if len(self.row_lower) != m or len(self.row_upper) != m:
            raise ValueError("ModelIR: row_lower/row_upper size != num_rows")
        if len(self.col_idx) != len(self.values) or int(self.row_ptr[-1]) != len(self.values):
            raise ValueError("ModelIR: row_ptr.back() must equal nnz")

    def numVars(self) -> int:  # noqa: N802 - reference naming
        return len(self.obj_coeffs)

    def numRows(self) -> int:  # noqa: N802
        return len(self.row_ptr) - 1

    def nnz(self) -> int:
        return len(self.values)

    def c_struct(self) -> L.CLp:
        lp = L.CLp()
        lp.num_rows, lp.num_cols, lp.nnz = self.numRows(), self.numVars(), self.nnz()
        lp.obj_sense, lp.obj_offset = int(self.obj_sense), float(self.obj_offset)
        lp.obj_coeffs = _ptr(self.obj_coeffs)
        lp.row_ptr = _ptr(self.row_ptr)
        lp.col_idx = _ptr(self.col_idx)
        lp.values = _ptr(self.values)
        lp.row_lower, lp.row_upper = _ptr(self.row_lower), _ptr(self.row_upper)
        lp.var_lower, lp.var_upper = _ptr(self.var_lower), _ptr(self.var_upper)
        return lp

    def multiply(self, x) -> np.ndarray:
        """FP64 A x (CSRMatrix::multiply) on the host, for checks."""
        x = _f64(x)
        rows = np.repeat(np.arange(self.numRows()), np.diff(self.row_ptr))
        return np.bincount(rows, weights=self.values * x[self.col_idx], minlength=self.numRows())


@dataclass
class PdhgOptions:
    """pramaan::gpu::PdhgOptions (include/pramaan/gpu/pdhg_solver.hpp:9-13)
    plus extensions whose defaults reproduce the reference."""
    tolerance: float = 1e-6
    max_iterations: int = 100000
    check_frequency: int = 100
    algorithm: int = 0          # 0: the reference iteration, 1: adaptive (PDLP-style), 2: Halpern
    termination: int | None = None  # default: reference criterion / relative KKT (adaptive)
    device: int = 0
    use_graph: bool = True
    profile_kernels: bool = False
    refine: bool = True         # adaptive mode: FP64 master iterates + FP32 corrections
    persistent: int = 0         # Halpern mode: 0 one cluster per LP runs each check interval when every LP
                                # has <= 2^20 non-zeros (else -1), 2 the cluster kernel always,
                                # 1 one cooperative kernel per interval, -1 two dependent launches
                                # per iteration in a CUDA graph
    gather_cache: int = 0       # 0: hot gather targets of large skewed operands in shared memory and
                                # L1-cached gathers where the autotuner finds them faster;
                                # 1: L1-cached gathers on every operand without hot slots; -1: plain
    launch_blocks: int = 0      # 0: autotuned blocks per SM of the large-operand products; > 0: fixed
    panel_split: int = 0        # reference algorithm, A x̄: 0 long rows of a power-law A over column
                                # panels held in shared memory (automatic), 1 whenever feasible,
                                # >= 2 with rows of that many entries as long rows, -1 tiled only

    def c_struct(self) -> L.COptions:
        o = L.COptions()
        L.lib().pramaan_pdhg_default_options(C.byref(o))
        o.tolerance = float(self.tolerance)
        o.max_iterations = int(self.max_iterations)
        o.check_frequency = int(self.check_frequency)
        o.algorithm = int(self.algorithm)
        if self.termination is None:
            o.termination = TERM_REFERENCE if int(self.algorithm) == ALGO_REFERENCE else TERM_RELATIVE_KKT
        else:
            o.termination = int(self.termination)
        o.device = int(self.device)
        o.use_graph = int(bool(self.use_graph))
        o.profile_kernels = int(bool(self.profile_kernels))
        o.refine = int(bool(self.refine))
        o.persistent = int(self.persistent)
        o.gather_cache = int(self.gather_cache)
        o.launch_blocks = int(self.launch_blocks)
        o.panel_split = int(self.panel_split)
        return o


@dataclass
class SolveResult:
    """pramaan::SolveResult (include/pramaan/simplex.hpp:40-76) + the dual y."""
    status: SolveStatus = SolveStatus.kIterationLimit
    x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    primal_residual: float = float("inf")
    dual_residual: float = float("inf")
    objective_value: float = 0.0
    row_activity: np.ndarray = field(default_factory=lambda: np.zeros(0))
    iterations: int = 0
    y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    restarts: int = 0
    checks: int = 0
    solve_ms: float = 0.0
    rel_primal: float = float("nan")
    rel_dual: float = float("nan")
    rel_gap: float = float("nan")
    primal_weight: float = 1.0
    step_size: float = 1.0
    compactions: int = 0        # batch solves: operand rebuilds during the batch


class PdhgSolver:
    """pramaan::gpu::PdhgSolver (include/pramaan/gpu/pdhg_solver.hpp:15-24)."""

    def __init__(self, options: PdhgOptions | None = None):
        self.options = options or PdhgOptions()

    def solve(self, model: ModelIR) -> SolveResult:
        n, m = model.numVars(), model.numRows()
        res = SolveResult()
        # Early returns of the reference keep x empty (src/gpu/pdhg_solver.cu:179-192).
        if n == 0:
            res.status = SolveStatus.kOptimal
            res.objective_value = model.obj_offset
            res.row_activity = np.zeros(m)
            res.iterations = 0
            return res
        if not np.all(np.isfinite(model.obj_coeffs)):
            res.status = SolveStatus.kNumericalFailure
            return res
        x = np.zeros(n)
        act = np.zeros(m)
        y = np.zeros(m)
        cr = L.CResult()
        cr.x, cr.row_activity, cr.y = _ptr(x), _ptr(act), _ptr(y)
        lp = model.c_struct()
        opt = self.options.c_struct()
        L.check(L.lib().pramaan_pdhg_solve(C.byref(lp), C.byref(opt), C.byref(cr)))
        res.status = SolveStatus(cr.status)
        res.iterations = cr.iterations
        res.primal_residual = cr.primal_residual
        res.dual_residual = cr.dual_residual
        res.objective_value = cr.objective_value
        res.x, res.row_activity, res.y = x, act, y
        res.restarts, res.checks, res.solve_ms = cr.restarts, cr.checks, cr.solve_ms
        res.rel_primal, res.rel_dual, res.rel_gap = cr.rel_primal, cr.rel_dual, cr.rel_gap
        res.primal_weight, res.step_size = cr.primal_weight, cr.step_size
        return res

    def solve_batch(self, models: list[ModelIR]) -> list[SolveResult]:
        """Solves many LPs in one packed launch sequence (pramaan_pdhg_solve_batch).

        Uses the Halpern algorithm when ``options.algorithm`` is ALGO_HALPERN and
        the adaptive algorithm otherwise, with relative-KKT termination; each LP
        keeps its own step size, weight, restarts and termination.
        """
        return solve_batch(models, self.options)


def solve_batch(models: list[ModelIR], options: PdhgOptions | None = None,
                warm: list | None = None) -> list[SolveResult]:
    """Batched PDHG over ``models`` (see ``PdhgSolver.solve_batch``).

    ``warm`` (optional) gives each LP a starting point: an object with
    attributes ``x``, ``y`` (arrays or None) and ``primal_weight`` (a float,
    <= 0 for the default), or None for a cold start
    (pramaan_pdhg_solve_batch_warm)."""
    opts = options or PdhgOptions()
    o = opts.c_struct()
    o.algorithm = ALGO_HALPERN if int(opts.algorithm) == ALGO_HALPERN else ALGO_ADAPTIVE
    o.termination = TERM_RELATIVE_KKT
    k = len(models)
    lps = (L.CLp * max(k, 1))()
    res = (L.CResult * max(k, 1))()
    keep = []
    outs = []
    for i, model in enumerate(models):
        lps[i] = model.c_struct()
        keep.append(model)
        x, act, y = np.zeros(model.numVars()), np.zeros(model.numRows()), np.zeros(model.numRows())
        res[i].x, res[i].row_activity, res[i].y = _ptr(x), _ptr(act), _ptr(y)
        outs.append((x, act, y))
    wptr = None
    if warm is not None:
        if len(warm) != k:
            raise ValueError("solve_batch: warm must have one entry per model")
        ws = (L.CWarmStart * max(k, 1))()
        for i, w in enumerate(warm):
            if w is None:
                ws[i].x, ws[i].y, ws[i].primal_weight = None, None, 0.0
                continue
            wx = None if getattr(w, "x", None) is None else _f64(w.x)
            wy = None if getattr(w, "y", None) is None else _f64(w.y)
            if wx is not None and len(wx) != models[i].numVars():
                raise ValueError("solve_batch: warm x has the wrong length")
            if wy is not None and len(wy) != models[i].numRows():
                raise ValueError("solve_batch: warm y has the wrong length")
            keep.extend([wx, wy])
            ws[i].x, ws[i].y = _ptr(wx), _ptr(wy)
            ws[i].primal_weight = float(getattr(w, "primal_weight", 0.0) or 0.0)
        wptr = ws
    L.check(L.lib().pramaan_pdhg_solve_batch_warm(lps, k, C.byref(o), wptr, res))
    out = []
    for i in range(k):
        cr = res[i]
        r = SolveResult()
        r.status = SolveStatus(cr.status)
        r.iterations = cr.iterations
        r.primal_residual, r.dual_residual = cr.primal_residual, cr.dual_residual
        r.objective_value = cr.objective_value
        r.x, r.row_activity, r.y = outs[i]
        if models[i].numVars() == 0:
            r.x = np.zeros(0)
        r.restarts, r.checks, r.solve_ms = cr.restarts, cr.checks, cr.solve_ms
        r.rel_primal, r.rel_dual, r.rel_gap = cr.rel_primal, cr.rel_dual, cr.rel_gap
        r.primal_weight, r.step_size = cr.primal_weight, cr.step_size
        r.compactions = int(cr.compactions)
        out.append(r)
    return out


# ---- test-harness launchers (src/gpu/pdhg.cu:77-241) ------------------------

def launch_spmv(row_ptr, col_idx, values, x, m: int, n: int) -> np.ndarray:
    """y = A x on the GPU (returns an empty array when m == 0)."""
    rp, ci, v, xx = _i32(row_ptr), _i32(col_idx), _f32(values), _f32(x)
    if m == 0:
        return np.zeros(0, np.float32)
    y = np.zeros(m, np.float32)
    L.check(L.lib().pramaan_launch_spmv(_ptr(rp), _ptr(ci), _ptr(v), len(v), _ptr(xx), _ptr(y), m, n))
    return y


def launch_spmv_t(row_ptr, col_idx, values, x, m: int, n: int) -> np.ndarray:
    """y = A^T x on the GPU (zeros when m == 0)."""
    rp, ci, v, xx = _i32(row_ptr), _i32(col_idx), _f32(values), _f32(x)
    y = np.zeros(n, np.float32)
    if n == 0:
        return y
    L.check(L.lib().pramaan_launch_spmv_t(_ptr(rp), _ptr(ci), _ptr(v), len(v), _ptr(xx), _ptr(y), m, n))
    return y


def launch_pdhg_iteration(x: np.ndarray, y: np.ndarray, gradient, Ax_bar, b,  # noqa: N803
                          tau: float, sigma: float) -> None:
    """One Step-1 iteration; x and y (float32 arrays) are updated in place."""
    assert x.dtype == np.float32 and y.dtype == np.float32
    g, ax, bb = _f32(gradient), _f32(Ax_bar), _f32(b)
    L.check(L.lib().pramaan_launch_pdhg_iteration(
        _ptr(x), _ptr(y), _ptr(g), _ptr(ax), _ptr(bb), len(x), len(y), float(tau), float(sigma)))


def release_cached_memory(device: int = -1) -> None:
    """Returns the device memory the library keeps for reuse to the driver
    (pramaan_release_cached_memory; -1: every device)."""
    L.check(L.lib().pramaan_release_cached_memory(int(device)))


class Session:
    """Device-resident solver state (pramaan_session_* entry points)."""

    def __init__(self, model: ModelIR, options: PdhgOptions | None = None):
        self.model = model
        self.options = options or PdhgOptions()
        self._h = C.c_void_p()
        lp = model.c_struct()
        opt = self.options.c_struct()
        L.check(L.lib().pramaan_session_create(C.byref(lp), C.byref(opt), C.byref(self._h)))

    def close(self) -> None:
        if self._h:
            L.check(L.lib().pramaan_session_destroy(self._h))
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def iterate(self, k: int) -> None:
        L.check(L.lib().pramaan_session_iterate(self._h, int(k)))

    def synchronize(self) -> None:
        L.check(L.lib().pramaan_session_synchronize(self._h))

    def residuals(self) -> tuple[float, float]:
        pv, dv = C.c_double(), C.c_double()
        L.check(L.lib().pramaan_session_residuals(self._h, C.byref(pv), C.byref(dv)))
        return pv.value, dv.value

    def iterates(self) -> tuple[np.ndarray, np.ndarray]:
        x = np.zeros(self.model.numVars(), np.float32)
        y = np.zeros(self.model.numRows(), np.float32)
        L.check(L.lib().pramaan_session_get_iterates(self._h, _ptr(x), _ptr(y)))
        return x, y

    def stream(self) -> int:
        return int(L.lib().pramaan_session_stream(self._h) or 0)

    def kernel_times(self, reset: bool = False) -> tuple[float, float, int]:
        a, b, n = C.c_double(), C.c_double(), C.c_int64()
        L.check(L.lib().pramaan_session_kernel_times(self._h, C.byref(a), C.byref(b), C.byref(n),
                                                     int(reset)))
        return a.value, b.value, n.value

    def kernel_bytes(self) -> tuple[float, float]:
        a, b = C.c_double(), C.c_double()
        L.check(L.lib().pramaan_session_kernel_bytes(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def gather_info(self) -> dict:
        """Gather modes of the dual product's operand A and the primal
        product's operand A^T: hot gather slots (0: no shared-memory copy) and
        whether the gathers are cached in L1, and the autotuned resident
        blocks per SM (0: default grid)."""
        v = [C.c_int32() for _ in range(6)]
        L.check(L.lib().pramaan_session_gather_info(self._h, *(C.byref(q) for q in v)))
        return {"A": {"hot_slots": v[0].value, "l1": bool(v[2].value), "blocks_per_sm": v[4].value},
                "AT": {"hot_slots": v[1].value, "l1": bool(v[3].value), "blocks_per_sm": v[5].value}}

    def panel_info(self) -> dict:
        """Column-panel split of the products: panels (0: the tiled A x̄
        alone), long rows of A x̄, their non-zeros and the row length from
        which a row is long; the hot rows of Aᵀy (0: the tiled Aᵀy alone)
        and their non-zeros."""
        p, lr, ml, hr = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        nz, hz = C.c_int64(), C.c_int64()
        L.check(L.lib().pramaan_session_panel_info(self._h, C.byref(p), C.byref(lr), C.byref(nz), C.byref(ml),
                                                   C.byref(hr), C.byref(hz)))
        return {"panels": p.value, "long_rows": lr.value, "long_nnz": nz.value, "min_len": ml.value,
                "primal_hot_rows": hr.value, "primal_hot_nnz": hz.value}

    def gather_slots(self) -> tuple[int, int]:
        """Hot gather slots of A and A^T."""
        g = self.gather_info()
        return g["A"]["hot_slots"], g["AT"]["hot_slots"]
