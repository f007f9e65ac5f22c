"""ctypes binding of libpramaan_b200.so (the C ABI in include/pramaan_b200.h).

Loading fails loudly: there is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libpramaan_b200.so"

PRAMAAN_OK = 0
PRAMAAN_ERR_INVALID_ARGUMENT = -1
PRAMAAN_ERR_CUDA = -2
PRAMAAN_ERR_DEVICE_TIMEOUT = -3
PRAMAAN_ERR_INTERNAL = -4

i32 = C.c_int32
i64 = C.c_int64
f64 = C.c_double
f32 = C.c_float
P = C.c_void_p


class CLp(C.Structure):
    _fields_ = [
        ("num_rows", i32), ("num_cols", i32), ("nnz", i32), ("obj_sense", i32),
        ("obj_offset", f64),
        ("obj_coeffs", P), ("row_ptr", P), ("col_idx", P), ("values", P),
        ("row_lower", P), ("row_upper", P), ("var_lower", P), ("var_upper", P),
    ]


class COptions(C.Structure):
    _fields_ = [
        ("tolerance", f64), ("max_iterations", i32), ("check_frequency", i32),
        ("algorithm", i32), ("termination", i32), ("device", i32), ("use_graph", i32),
        ("profile_kernels", i32), ("refine", i32), ("reserved_d", f64),
        ("persistent", i32), ("gather_cache", i32), ("launch_blocks", i32), ("panel_split", i32), ("reserved", i32 * 2),
    ]


class CResult(C.Structure):
    _fields_ = [
        ("status", i32), ("iterations", i32),
        ("primal_residual", f64), ("dual_residual", f64), ("objective_value", f64),
        ("x", P), ("row_activity", P), ("y", P),
        ("restarts", i32), ("checks", i32), ("solve_ms", f64),
        ("rel_primal", f64), ("rel_dual", f64), ("rel_gap", f64), ("primal_weight", f64),
        ("step_size", f64), ("compactions", f64),
    ]


class CWarmStart(C.Structure):
    _fields_ = [("x", P), ("y", P), ("primal_weight", f64)]


class CLadderOptions(C.Structure):
    _fields_ = [("residual_threshold", f64), ("gpu_max_iterations", i32), ("gpu_check_frequency", i32),
                ("gpu_tolerance", f64), ("refine", i32), ("refine_max_iterations", i32),
                ("refine_tolerance", f64), ("device", i32), ("reserved", i32 * 3)]


class CLadderResult(C.Structure):
    _fields_ = [("stage", i32), ("escalation_reason", i32), ("refine_escalation_reason", i32),
                ("gpu_status", i32), ("gpu_iterations", i32), ("refine_status", i32),
                ("refine_iterations", i32), ("reserved", i32),
                ("gpu_primal_residual", f64), ("gpu_dual_residual", f64), ("gpu_objective", f64),
                ("gpu_elapsed_ms", f64), ("refine_primal_residual", f64), ("refine_dual_residual", f64),
                ("refine_objective", f64), ("refine_elapsed_ms", f64), ("rel_primal", f64),
                ("rel_dual", f64), ("rel_gap", f64), ("objective_value", f64), ("total_elapsed_ms", f64),
                ("x", P), ("y", P), ("row_activity", P)]


class CCertificate(C.Structure):
    _fields_ = [("objective_value", f64), ("primal_residual", f64), ("bound_violation", f64),
                ("rel_primal", f64), ("rel_dual", f64), ("rel_gap", f64),
                ("primal_objective", f64), ("dual_objective", f64), ("kkt", f64)]


# (name, restype, argtypes) for every entry point declared in the header.
SIGNATURES = [
    ("pramaan_version", C.c_char_p, []),
    ("pramaan_last_error", C.c_char_p, []),
    ("pramaan_pdhg_default_options", None, [C.POINTER(COptions)]),
    ("pramaan_pdhg_solve", C.c_int, [C.POINTER(CLp), C.POINTER(COptions), C.POINTER(CResult)]),
    ("pramaan_pdhg_solve_batch", C.c_int, [C.POINTER(CLp), i32, C.POINTER(COptions), C.POINTER(CResult)]),
    ("pramaan_pdhg_solve_batch_warm", C.c_int,
     [C.POINTER(CLp), i32, C.POINTER(COptions), C.POINTER(CWarmStart), C.POINTER(CResult)]),
    ("pramaan_ladder_default_options", None, [C.POINTER(CLadderOptions)]),
    ("pramaan_ladder_solve", C.c_int, [C.POINTER(CLp), C.POINTER(CLadderOptions), C.POINTER(CLadderResult)]),
    ("pramaan_certify_batch", C.c_int,
     [C.POINTER(CLp), i32, C.POINTER(CWarmStart), i32, i32, C.POINTER(CCertificate)]),
    ("pramaan_gnn_num_params", i32, []),
    ("pramaan_gnn_create", C.c_int, [i32, C.c_uint64, C.POINTER(P)]),
    ("pramaan_gnn_destroy", C.c_int, [P]),
    ("pramaan_gnn_get_params", C.c_int, [P, P]),
    ("pramaan_gnn_set_params", C.c_int, [P, P]),
    ("pramaan_gnn_graph_create", C.c_int,
     [C.POINTER(CLp), i32, C.POINTER(CWarmStart), C.POINTER(CWarmStart), i32, C.POINTER(P)]),
    ("pramaan_gnn_graph_destroy", C.c_int, [P]),
    ("pramaan_gnn_predict", C.c_int, [P, P, P, P, P]),
    ("pramaan_gnn_gradients", C.c_int, [P, P, P, C.POINTER(f64)]),
    ("pramaan_gnn_train_step", C.c_int, [P, P, f32, C.POINTER(f64)]),
    ("pramaan_gnn_trace_size", i64, [P]),
    ("pramaan_gnn_forward_trace", C.c_int, [P, P, P]),
    ("pramaan_launch_spmv", C.c_int, [P, P, P, i32, P, P, i32, i32]),
    ("pramaan_launch_spmv_t", C.c_int, [P, P, P, i32, P, P, i32, i32]),
    ("pramaan_launch_pdhg_iteration", C.c_int, [P, P, P, P, P, i32, i32, f32, f32]),
    ("pramaan_spmv_noalloc", C.c_int, [P, P, P, i32, i32, i32, P, P, P]),
    ("pramaan_session_create", C.c_int, [C.POINTER(CLp), C.POINTER(COptions), C.POINTER(P)]),
    ("pramaan_session_destroy", C.c_int, [P]),
    ("pramaan_session_iterate", C.c_int, [P, i32]),
    ("pramaan_session_synchronize", C.c_int, [P]),
    ("pramaan_session_residuals", C.c_int, [P, C.POINTER(f64), C.POINTER(f64)]),
    ("pramaan_session_get_iterates", C.c_int, [P, P, P]),
    ("pramaan_session_stream", P, [P]),
    ("pramaan_session_kernel_times", C.c_int,
     [P, C.POINTER(f64), C.POINTER(f64), C.POINTER(i64), i32]),
    ("pramaan_session_kernel_bytes", C.c_int, [P, C.POINTER(f64), C.POINTER(f64)]),
    ("pramaan_session_gather_info", C.c_int, [P] + [C.POINTER(i32)] * 6),
    ("pramaan_session_panel_info", C.c_int, [P, C.POINTER(i32), C.POINTER(i32), C.POINTER(C.c_int64),
                                             C.POINTER(i32), C.POINTER(i32), C.POINTER(C.c_int64)]),
    ("pramaan_release_cached_memory", C.c_int, [i32]),
    ("pramaan_measure_gather_rate", C.c_int, [P, i32, i32, i32, C.POINTER(f64)]),
]

_lib: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m pramaan_b200.build` "
                "(the CUDA library is required; there is no CPU fallback)")
        h = C.CDLL(str(LIB_PATH))
        for name, res, args in SIGNATURES:
            fn = getattr(h, name)
            fn.restype = res
            fn.argtypes = args
        _lib = h
    return _lib


class PramaanError(RuntimeError):
    """A failed library call (CUDA error, device timeout, internal error)."""

    def __init__(self, code: int, msg: str):
        super().__init__(msg)
        self.code = code


def check(rc: int) -> None:
    if rc == PRAMAAN_OK:
        return
    msg = (lib().pramaan_last_error() or b"").decode(errors="replace")
    if rc == PRAMAAN_ERR_INVALID_ARGUMENT:
        raise ValueError(msg)
    raise PramaanError(rc, msg)
