"""The CUDA path against golden vectors recorded from the reference's own
GPU PDHG on a B200 (tests/golden/make_ref_golden.py), through the C ABI.

Tolerances follow the reference's own GPU tests: SpMV elements within
1e-4 + 1e-4 |y| (tests/test_gpu_pdhg.cpp:191-193) — the products here are
summed in another (deterministic) order, so they agree to a few ulps; the
step kernel bit-identically (both fuse the same multiply-adds); solves with
the same status, the same iteration count up to the check that stops them
(at most 10% apart), objective within 1e-4 (1 + |obj|)
(tests/test_gpu_pdhg.cpp:444-447) and x within 1e-3.
"""
from __future__ import annotations

import numpy as np
import pytest

from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus
from pramaan_b200.pdhg import launch_pdhg_iteration, launch_spmv, launch_spmv_t
from test_golden_reference import GOLDEN, golden_model, iterations_agree, solve_cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g():
    return np.load(GOLDEN)


def test_spmv_pair_matches_reference_gpu(g):
    for i in range(5):
        p = f"spmv/case{i}/"
        m, n = (int(v) for v in g[p + "dims"])
        y = launch_spmv(g[p + "row_ptr"], g[p + "col_idx"], g[p + "values"], g[p + "x"], m, n)
        ref = g[p + "y"]
        assert np.all(np.abs(y - ref) <= 1e-4 + 1e-4 * np.abs(ref))
        yt = launch_spmv_t(g[p + "row_ptr"], g[p + "col_idx"], g[p + "values"], g[f"spmv_t/case{i}/yin"], m, n)
        ref_t = g[f"spmv_t/case{i}/out"]
        assert np.all(np.abs(yt - ref_t) <= 1e-4 + 1e-4 * np.abs(ref_t))


def test_step_bit_identical_to_reference_gpu(g):
    for i in range(3):
        p = f"step/case{i}/"
        tau, sig = (float(v) for v in g[p + "tau_sigma"])
        x, y = g[p + "x"].copy(), g[p + "y"].copy()
        launch_pdhg_iteration(x, y, g[p + "g"], g[p + "ax"], g[p + "b"], tau, sig)
        np.testing.assert_array_equal(x.view(np.uint32), g[p + "x_out"].view(np.uint32))
        np.testing.assert_array_equal(y.view(np.uint32), g[p + "y_out"].view(np.uint32))


def test_solve_matches_reference_gpu_solve(g):
    for case in solve_cases(g):
        p = f"solve/{case}/"
        model = golden_model(g, case)
        tol, max_it, cf = g[p + "opts"]
        r = PdhgSolver(PdhgOptions(tolerance=float(tol), max_iterations=int(max_it),
                                   check_frequency=int(cf))).solve(model)
        ref_obj = float(g[p + "objective_value"])
        assert int(r.status) == int(g[p + "status"]), case
        assert iterations_agree(r.iterations, int(g[p + "iterations"]), int(cf)), (case, r.iterations)
        assert abs(r.objective_value - ref_obj) <= 1e-4 * (1 + abs(ref_obj)), case
        if model.numVars():
            assert np.max(np.abs(r.x - g[p + "x"])) <= 1e-3, case
            if r.status == SolveStatus.kOptimal:
                np.testing.assert_allclose(r.row_activity, g[p + "row_activity"], rtol=1e-3, atol=1e-3)
