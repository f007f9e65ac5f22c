"""Pins the oracle to golden vectors recorded from the reference's own GPU
PDHG (src/gpu/pdhg_solver.cu, src/gpu/pdhg.cu built for sm_100a from the
reference's sources and run on a B200 by tests/golden/make_ref_golden.py).

* launch_spmv (row-per-thread sums, src/gpu/pdhg_kernels.cuh:24-37): the
  oracle's fused-multiply-add row sums are bit-identical;
* launch_pdhg_iteration (src/gpu/pdhg.cu:77-150): bit-identical;
* launch_spmv_t: the reference scatters with atomicAdd
  (src/gpu/pdhg_kernels.cuh:42-54), so its summation order is not defined;
  compared within 1e-5 relative (plus 1e-6 of the column's magnitude);
* PdhgSolver::solve on the known-answer LPs, three seeded random LPs and
  afiro: the same status; the same iteration count (the check that stops a
  solve can move by a few check intervals because Aᵀy's order differs; at
  most 10% of the count); objective within 1e-4 * (1 + |obj|); x within
  1e-3 absolute.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

import oracle
from pramaan_b200.pdhg import ModelIR

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_gpu_golden.npz"


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def solve_cases(g):
    return sorted({k.split("/")[1] for k in g.files if k.startswith("solve/")})


def golden_model(g, case: str) -> ModelIR:
    p = f"solve/{case}/lp_"
    return ModelIR(g[p + "c"], g[p + "row_ptr"], g[p + "col_idx"], g[p + "values"], g[p + "row_lower"],
                   g[p + "row_upper"], g[p + "var_lower"], g[p + "var_upper"], int(g[p + "obj_sense"]),
                   float(g[p + "obj_offset"]))


def iterations_agree(mine: int, ref: int, cf: int) -> bool:
    return abs(mine - ref) <= max(2 * cf, 0.1 * ref)


def test_golden_file_holds_every_case(g):
    assert {"afiro", "wyndor", "multi", "random_0", "random_1", "random_2"} <= set(solve_cases(g))
    assert sum(k.startswith("spmv/") and k.endswith("/y") for k in g.files) == 5
    assert sum(k.startswith("step/") and k.endswith("/x_out") for k in g.files) == 3


def test_oracle_spmv_bit_identical_to_reference_gpu(g):
    for i in range(5):
        p = f"spmv/case{i}/"
        m = int(g[p + "dims"][0])
        y = oracle.spmv_f32_fma(g[p + "row_ptr"], g[p + "col_idx"], g[p + "values"], g[p + "x"], m)
        np.testing.assert_array_equal(y.view(np.uint32), g[p + "y"].view(np.uint32))


def test_oracle_spmv_t_matches_reference_gpu_scatter(g):
    for i in range(5):
        p = f"spmv/case{i}/"
        m, n = (int(v) for v in g[p + "dims"])
        yin = g[f"spmv_t/case{i}/yin"]
        ref = g[f"spmv_t/case{i}/out"]
        yt = oracle.spmv_t_f32(g[p + "row_ptr"], g[p + "col_idx"], g[p + "values"], yin, m, n)
        # |A|^T |y| bounds the rounding of any summation order
        absA = oracle.spmv_t_f32(g[p + "row_ptr"], g[p + "col_idx"], np.abs(g[p + "values"]), np.abs(yin), m, n)
        assert np.all(np.abs(yt - ref) <= 1e-5 * np.abs(ref) + 1e-6 * absA + 1e-30)


def test_oracle_step_bit_identical_to_reference_gpu(g):
    for i in range(3):
        p = f"step/case{i}/"
        tau, sig = g[p + "tau_sigma"]
        xo, yo = oracle.step1(g[p + "x"], g[p + "y"], g[p + "g"], g[p + "ax"], g[p + "b"], tau, sig, use_fma=True)
        np.testing.assert_array_equal(xo.view(np.uint32), g[p + "x_out"].view(np.uint32))
        np.testing.assert_array_equal(yo.view(np.uint32), g[p + "y_out"].view(np.uint32))


def test_oracle_solve_matches_reference_gpu_solve(g):
    for case in solve_cases(g):
        p = f"solve/{case}/"
        model = golden_model(g, case)
        tol, max_it, cf = g[p + "opts"]
        r = oracle.solve_ref(model, tol=float(tol), max_iterations=int(max_it), check_frequency=int(cf))
        ref_obj = float(g[p + "objective_value"])
        assert r["status"] == int(g[p + "status"]), case
        assert iterations_agree(r["iterations"], int(g[p + "iterations"]), int(cf)), (case, r["iterations"])
        assert abs(r["objective_value"] - ref_obj) <= 1e-4 * (1 + abs(ref_obj)), case
        if model.numVars():
            assert np.max(np.abs(r["x"] - g[p + "x"])) <= 1e-3, case
