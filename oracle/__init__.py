"""Oracle for libpramaan_b200 — TEST INFRASTRUCTURE ONLY.

* ``orc``: ctypes binding of ``_build/liborc.so``, the C restatement of the
  reference's GPU PDHG path (``pdhg_oracle.c``).
* ``ref_cpu`` / ``ref_gpu``: the reference's own solvers compiled from its
  sources into ``_ref/`` (when that build exists).

Only tests/, ``__graft_entry__.smoke()`` and the cpu_baseline leg of bench.py
use this package, and only to check or time beside the CUDA library.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORC_PATH = HERE / "_build" / "liborc.so"
REF_CPU_PATH = HERE / "_ref" / "libref_cpu.so"
REF_GPU_PATH = HERE / "_ref" / "libref_gpu.so"

i32, f64, f32, P = C.c_int32, C.c_double, C.c_float, C.c_void_p


class OrcLp(C.Structure):
    _fields_ = [
        ("m", i32), ("n", i32), ("nnz", i32), ("obj_sense", i32), ("obj_offset", f64),
        ("c", P), ("row_ptr", P), ("col_idx", P), ("values", P),
        ("row_lower", P), ("row_upper", P), ("var_lower", P), ("var_upper", P),
    ]


class OrcResult(C.Structure):
    _fields_ = [
        ("status", i32), ("iterations", i32), ("restarts", i32), ("checks", i32),
        ("primal_residual", f64), ("dual_residual", f64), ("objective_value", f64),
        ("x", P), ("row_activity", P), ("y", P), ("x32", P),
    ]


class RefResult(C.Structure):
    _fields_ = [
        ("status", i32), ("iterations", i32), ("crash_basis_pivots", i32), ("reserved", i32),
        ("primal_residual", f64), ("dual_residual", f64), ("objective_value", f64),
        ("x", P), ("row_activity", P),
    ]


def ptr(a):
    return None if a is None or a.size == 0 else a.ctypes.data_as(C.c_void_p)


_orc = None


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORC_PATH.exists():
            from . import build as _b
            _b.build_oracle()
        h = C.CDLL(str(ORC_PATH))
        sig = {
            "orc_spmv_f32": [i32, P, P, P, P, P],
            "orc_spmv_f32_fma": [i32, P, P, P, P, P],
            "orc_spmv_t_f32": [i32, i32, P, P, P, P, P],
            "orc_spmv_f64": [i32, P, P, P, P, P],
            "orc_transpose_f32": [i32, i32, P, P, P, P, P, P],
            "orc_dual_update": [i32, P, P, P, P, P],
            "orc_primal_update": [i32, P, P, P, P, P, P, P],
            "orc_step1": [i32, P, P, f32, i32, P, P, P, f32, i32],
            "orc_step_sizes": [i32, i32, P, P, P, P, P],
            "orc_fp64_residuals": [C.POINTER(OrcLp), P, P, P, P, f64, C.POINTER(f64), C.POINTER(f64)],
            "orc_pdhg_trajectory": [C.POINTER(OrcLp), i32, P, P, P],
            "orc_pdhg_solve_ref": [C.POINTER(OrcLp), f64, i32, i32, C.POINTER(OrcResult)],
            "orc_certificate": [C.POINTER(OrcLp), P, C.POINTER(f64), C.POINTER(f64), C.POINTER(f64)],
            "orc_rel_kkt": [C.POINTER(OrcLp), P, P, P],
            "orc_num_threads": [],
            "orc_set_num_threads": [i32],
            "orc_pdhg_iterations_mt": [i32, i32, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, P, i32],
        }
        for name, args in sig.items():
            fn = getattr(h, name)
            fn.argtypes = args
            fn.restype = i32 if name == "orc_num_threads" else None
        _orc = h
    return _orc


def lp_struct(model) -> OrcLp:
    """OrcLp view of a pramaan_b200.ModelIR (arrays must stay alive)."""
    lp = OrcLp()
    lp.m, lp.n, lp.nnz = model.numRows(), model.numVars(), model.nnz()
    lp.obj_sense, lp.obj_offset = int(model.obj_sense), float(model.obj_offset)
    lp.c, lp.row_ptr, lp.col_idx, lp.values = (ptr(model.obj_coeffs), ptr(model.row_ptr),
                                                ptr(model.col_idx), ptr(model.values))
    lp.row_lower, lp.row_upper = ptr(model.row_lower), ptr(model.row_upper)
    lp.var_lower, lp.var_upper = ptr(model.var_lower), ptr(model.var_upper)
    return lp


# ---- convenience wrappers -----------------------------------------------------

def spmv_f32(rp, ci, v, x, m):
    y = np.zeros(m, np.float32)
    orc().orc_spmv_f32(m, ptr(rp), ptr(ci), ptr(v), ptr(x), ptr(y))
    return y


def spmv_f32_fma(rp, ci, v, x, m):
    """Row sums with one fused multiply-add per entry (the reference GPU kernel's arithmetic)."""
    y = np.zeros(m, np.float32)
    orc().orc_spmv_f32_fma(m, ptr(rp), ptr(ci), ptr(v), ptr(x), ptr(y))
    return y


def spmv_t_f32(rp, ci, v, x, m, n):
    y = np.zeros(n, np.float32)
    orc().orc_spmv_t_f32(m, n, ptr(rp), ptr(ci), ptr(v), ptr(x), ptr(y))
    return y


def step1(x, y, g, ax, b, tau, sigma, use_fma=True):
    x = np.array(x, np.float32)
    y = np.array(y, np.float32)
    orc().orc_step1(len(x), ptr(x), ptr(np.asarray(g, np.float32)), tau, len(y), ptr(y),
                    ptr(np.asarray(ax, np.float32)), ptr(np.asarray(b, np.float32)), sigma,
                    int(use_fma))
    return x, y


def step_sizes(model):
    v32 = model.values.astype(np.float32)
    sig = np.zeros(model.numRows(), np.float32)
    tau = np.zeros(model.numVars(), np.float32)
    orc().orc_step_sizes(model.numRows(), model.numVars(), ptr(model.row_ptr), ptr(model.col_idx),
                         ptr(v32), ptr(sig), ptr(tau))
    return sig, tau


def trajectory(model, iters: int):
    x = np.zeros(model.numVars(), np.float32)
    y = np.zeros(model.numRows(), np.float32)
    xb = np.zeros(model.numVars(), np.float32)
    lp = lp_struct(model)
    orc().orc_pdhg_trajectory(C.byref(lp), iters, ptr(x), ptr(y), ptr(xb))
    return x, y, xb


def residuals_ref(model, x32, y32, tol):
    """ComputeFp64Residuals on FP32 iterates."""
    lp = lp_struct(model)
    sgn = -1.0 if int(model.obj_sense) == 1 else 1.0
    c32 = (np.float32(sgn) * model.obj_coeffs).astype(np.float32)
    c32 = (sgn * model.obj_coeffs).astype(np.float32)
    v32 = model.values.astype(np.float32)
    pv, dv = f64(), f64()
    x32 = np.ascontiguousarray(x32, np.float32)
    y32 = np.ascontiguousarray(y32, np.float32)
    orc().orc_fp64_residuals(C.byref(lp), ptr(v32), ptr(c32), ptr(x32), ptr(y32), tol,
                             C.byref(pv), C.byref(dv))
    return pv.value, dv.value


def solve_ref(model, tol=1e-6, max_iterations=100000, check_frequency=100):
    """The reference solve restated on the CPU; returns a dict."""
    n, m = model.numVars(), model.numRows()
    x = np.zeros(n)
    act = np.zeros(m)
    y = np.zeros(m, np.float32)
    x32 = np.zeros(n, np.float32)
    r = OrcResult()
    r.x, r.row_activity, r.y, r.x32 = ptr(x), ptr(act), ptr(y), ptr(x32)
    lp = lp_struct(model)
    orc().orc_pdhg_solve_ref(C.byref(lp), tol, max_iterations, check_frequency, C.byref(r))
    return dict(status=r.status, iterations=r.iterations, restarts=r.restarts, checks=r.checks,
                primal_residual=r.primal_residual, dual_residual=r.dual_residual,
                objective_value=r.objective_value, x=x, row_activity=act, y=y, x32=x32)


def certificate(model, x):
    lp = lp_struct(model)
    o, p, b = f64(), f64(), f64()
    x = np.ascontiguousarray(x, np.float64)
    orc().orc_certificate(C.byref(lp), ptr(x), C.byref(o), C.byref(p), C.byref(b))
    return dict(objective=o.value, primal_residual=p.value, bound_violation=b.value)


def rel_kkt(model, x, y):
    lp = lp_struct(model)
    out = np.zeros(5)
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    orc().orc_rel_kkt(C.byref(lp), ptr(x), ptr(y), ptr(out))
    return dict(primal=out[0], dual=out[1], gap=out[2], pobj=out[3], dobj=out[4])


# ---- the reference's own solvers (oracle/_ref) --------------------------------

def _load_ref(path: Path, gpu: bool) -> C.CDLL | None:
    if not path.exists():
        return None
    h = C.CDLL(str(path))
    h.ref_last_error.restype = C.c_char_p
    h.ref_simplex_solve.argtypes = [C.POINTER(OrcLp), i32, f64, P, C.POINTER(RefResult)]
    h.ref_dual_simplex_solve.argtypes = [C.POINTER(OrcLp), i32, f64, C.POINTER(RefResult)]
    h.ref_ipm_solve.argtypes = [C.POINTER(OrcLp), i32, f64, C.POINTER(RefResult)]
    h.ref_mps_open.argtypes = [C.c_char_p, C.POINTER(P)]
    h.ref_mps_dims.argtypes = [P, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32), C.POINTER(i32),
                               C.POINTER(f64)]
    h.ref_mps_dims.restype = None
    h.ref_mps_fetch.argtypes = [P] * 9
    h.ref_mps_fetch.restype = None
    h.ref_mps_close.argtypes = [P]
    h.ref_mps_close.restype = None
    if gpu:
        h.ref_pdhg_solve.argtypes = [C.POINTER(OrcLp), f64, i32, i32, C.POINTER(RefResult)]
        h.ref_launch_spmv.argtypes = [P, P, P, i32, P, P, i32, i32]
        h.ref_launch_spmv_t.argtypes = [P, P, P, i32, P, P, i32, i32]
        h.ref_launch_pdhg_iteration.argtypes = [P, P, P, P, P, i32, i32, f32, f32]
    return h


_ref = {}


def ref_cpu() -> C.CDLL | None:
    if "cpu" not in _ref:
        _ref["cpu"] = _load_ref(REF_CPU_PATH, gpu=False)
    return _ref["cpu"]


def ref_gpu() -> C.CDLL | None:
    if "gpu" not in _ref:
        _ref["gpu"] = _load_ref(REF_GPU_PATH, gpu=True)
    return _ref["gpu"]


def ref_solve(kind: str, model, max_iterations=10000, tolerance=1e-9, hint=None,
              check_frequency=100, lib=None):
    """Runs one of the reference's solvers: 'simplex', 'dual', 'ipm' or 'pdhg'."""
    h = lib or (ref_gpu() if kind == "pdhg" else ref_cpu())
    if h is None:
        raise RuntimeError("oracle/_ref is not built")
    n, m = model.numVars(), model.numRows()
    x = np.full(n, np.nan)
    act = np.full(m, np.nan)
    r = RefResult()
    r.x, r.row_activity = ptr(x), ptr(act)
    lp = lp_struct(model)
    if kind == "simplex":
        hh = None if hint is None else np.ascontiguousarray(hint, np.float64)
        rc = h.ref_simplex_solve(C.byref(lp), max_iterations, tolerance, ptr(hh), C.byref(r))
    elif kind == "dual":
        rc = h.ref_dual_simplex_solve(C.byref(lp), max_iterations, tolerance, C.byref(r))
    elif kind == "ipm":
        rc = h.ref_ipm_solve(C.byref(lp), max_iterations, tolerance, C.byref(r))
    elif kind == "pdhg":
        rc = h.ref_pdhg_solve(C.byref(lp), tolerance, max_iterations, check_frequency, C.byref(r))
    else:
        raise ValueError(kind)
    if rc != 0:
        raise RuntimeError(h.ref_last_error().decode())
    return dict(status=r.status, iterations=r.iterations, crash_basis_pivots=r.crash_basis_pivots,
                primal_residual=r.primal_residual, dual_residual=r.dual_residual,
                objective_value=r.objective_value, x=x, row_activity=act)


def ref_load_mps(path: str):
    """Parses an MPS file with the reference's parser into a ModelIR."""
    from pramaan_b200.pdhg import ModelIR
    h = ref_cpu()
    if h is None:
        raise RuntimeError("oracle/_ref is not built")
    hd = P()
    if h.ref_mps_open(str(path).encode(), C.byref(hd)) != 0:
        raise RuntimeError(h.ref_last_error().decode())
    m, n, nnz, sense, off = i32(), i32(), i32(), i32(), f64()
    h.ref_mps_dims(hd, C.byref(m), C.byref(n), C.byref(nnz), C.byref(sense), C.byref(off))
    m, n, nnz = m.value, n.value, nnz.value
    c = np.zeros(n); rp = np.zeros(m + 1, np.int32); ci = np.zeros(nnz, np.int32)
    v = np.zeros(nnz); rl = np.zeros(m); ru = np.zeros(m); vl = np.zeros(n); vu = np.zeros(n)
    h.ref_mps_fetch(hd, ptr(c), ptr(rp), ptr(ci), ptr(v), ptr(rl), ptr(ru), ptr(vl), ptr(vu))
    h.ref_mps_close(hd)
    return ModelIR(c, rp, ci, v, rl, ru, vl, vu, sense.value, off.value)
