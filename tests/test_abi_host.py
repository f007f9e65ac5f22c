"""CPU-side checks of the C ABI: the library loads, exports every entry point
include/pramaan_b200.h declares, and its host-only functions behave (no GPU
compute is called here)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import pramaan_b200
from pramaan_b200 import _lib as L
from pramaan_b200.pdhg import ModelIR, PdhgOptions

HEADERS = sorted((Path(__file__).resolve().parent.parent / "include").glob("*.h"))


def declared_symbols():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        names.update(re.findall(r"PRAMAAN_API\s+[\w\s\*]+?\b(pramaan_\w+)\s*\(", text))
    return sorted(names)


def test_headers_declare_entry_points():
    syms = declared_symbols()
    assert "pramaan_pdhg_solve" in syms and "pramaan_launch_spmv" in syms
    assert len(syms) >= 16


def test_library_exports_every_declared_symbol(lib):
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_ctypes_binding_covers_header():
    bound = {name for name, _, _ in L.SIGNATURES}
    assert set(declared_symbols()) <= bound


def test_struct_layouts_match_header():
    # pramaan_lp: 4 int32 + double + 8 pointers; options 64 bytes; result.
    assert C.sizeof(L.CLp) == 4 * 4 + 8 + 8 * 8
    assert C.sizeof(L.COptions) == 8 + 4 * 8 + 8 + 4 * 6
    assert L.COptions.refine.offset == 36 and L.COptions.reserved_d.offset == 40
    # persistent, gather_cache, launch_blocks, panel_split, reserved[2] after reserved_d
    assert L.COptions.persistent.offset == 48 and L.COptions.launch_blocks.offset == 56
    assert L.COptions.panel_split.offset == 60
    assert L.CResult.restarts.offset == 8 + 3 * 8 + 3 * 8


def test_default_options_match_reference(lib):
    o = L.COptions()
    lib.pramaan_pdhg_default_options(C.byref(o))
    # include/pramaan/gpu/pdhg_solver.hpp:9-13
    assert o.tolerance == 1e-6 and o.max_iterations == 100000 and o.check_frequency == 100
    assert o.algorithm == 0 and o.termination == 0 and o.refine == 1
    assert o.persistent == 0 and o.gather_cache == 0 and o.launch_blocks == 0   # autotuned, automatic
    assert o.panel_split == 0   # column-panel splits chosen automatically
    p = PdhgOptions()
    assert (p.tolerance, p.max_iterations, p.check_frequency) == (1e-6, 100000, 100)


def test_version_and_error_strings(lib):
    assert b"sm_100a" in lib.pramaan_version()
    assert isinstance(lib.pramaan_last_error(), bytes)


def test_null_arguments_are_rejected_without_gpu(lib):
    assert lib.pramaan_pdhg_solve(None, None, None) == L.PRAMAAN_ERR_INVALID_ARGUMENT
    assert b"NULL" in lib.pramaan_last_error()
    assert lib.pramaan_session_iterate(None, 1) == L.PRAMAAN_ERR_INVALID_ARGUMENT


def test_trivial_no_variable_lp_needs_no_gpu():
    # n == 0 returns before any device work (src/gpu/pdhg_solver.cu:179-184).
    model = ModelIR([], [0, 0, 0], [], [], [1, 2], [3, 4], [], [], 0, 7.5)
    r = pramaan_b200.PdhgSolver().solve(model)
    assert r.status == pramaan_b200.SolveStatus.kOptimal
    assert r.objective_value == 7.5 and r.x.size == 0
    np.testing.assert_array_equal(r.row_activity, np.zeros(2))


def test_nonfinite_objective_is_numerical_failure_without_gpu():
    model = ModelIR([1.0, np.nan], [0, 2], [0, 1], [1.0, 1.0], [1], [1], [0, 0], [1, 1])
    r = pramaan_b200.PdhgSolver().solve(model)
    assert r.status == pramaan_b200.SolveStatus.kNumericalFailure and r.x.size == 0


def test_bad_options_rejected(lib):
    model = ModelIR([1.0], [0, 1], [0], [1.0], [1], [1], [0], [1])
    with pytest.raises(ValueError, match="check_frequency"):
        pramaan_b200.PdhgSolver(PdhgOptions(check_frequency=0)).solve(model)


def test_model_validation():
    with pytest.raises(ValueError):
        ModelIR([1.0], [0, 2], [0], [1.0], [1], [1], [0], [1])
    with pytest.raises(ValueError):
        ModelIR([1.0], [0, 1], [0], [1.0], [1, 2], [1], [0], [1])
