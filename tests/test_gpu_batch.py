"""GPU tests of the batched adaptive PDHG (pramaan_pdhg_solve_batch).

The batch has no reference counterpart; each LP of a batch is judged like a
single adaptive solve: the oracle's FP64 relative KKT (orc_rel_kkt) on the
returned (x, y) meets the tolerance, the reported KKT equals the oracle's
within 1e-4 relative, and the objective equals the same LP solved alone
(`pramaan_pdhg_solve`, adaptive) within 1e-4 * (1 + |obj|) at 1e-6 and
1e-7 * (1 + |obj|) at 1e-8.  Early answers (no variables, non-finite cost)
follow the reference (src/gpu/pdhg_solver.cu:179-192).
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN
from pramaan_b200 import ModelIR, PdhgOptions, PdhgSolver, SolveStatus, solve_batch
from pramaan_b200.generators import random_sparse_lp, rolling_horizon_batch, rolling_horizon_lp
from pramaan_b200.pdhg import ALGO_ADAPTIVE

pytestmark = pytest.mark.gpu


def opts(tol, max_it=300000):
    return PdhgOptions(tolerance=tol, max_iterations=max_it, check_frequency=64, algorithm=ALGO_ADAPTIVE)


def check(model, r, tol):
    k = oracle.rel_kkt(model, r.x, r.y)
    assert max(k["primal"], k["dual"], k["gap"]) <= tol * 1.0001, k
    for mine, theirs in ((r.rel_primal, k["primal"]), (r.rel_dual, k["dual"]), (r.rel_gap, k["gap"])):
        assert mine == pytest.approx(theirs, rel=1e-4, abs=1e-13)
    np.testing.assert_allclose(r.row_activity, model.multiply(r.x), rtol=1e-12, atol=1e-9)


def mixed_batch():
    models = [KNOWN[name][0] for name in ("wyndor", "multi", "bounded", "equality", "one_var")]
    models += [random_sparse_lp(60, 180, 4, seed=s) for s in range(3)]
    models += [rolling_horizon_lp(T, P, seed=T + P) for T, P in ((24, 5), (30, 8), (48, 6))]
    return models


def test_batch_matches_single_solves():
    models = mixed_batch()
    res = solve_batch(models, opts(1e-6))
    assert len(res) == len(models)
    for model, r in zip(models, res):
        assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
        check(model, r, 1e-6)
        alone = PdhgSolver(opts(1e-6)).solve(model)
        assert alone.status == SolveStatus.kOptimal
        assert r.objective_value == pytest.approx(alone.objective_value, rel=1e-4, abs=1e-4)


def test_batch_known_objectives():
    names = ["wyndor", "multi", "bounded", "equality", "one_var", "zero_obj", "sparse_zeros"]
    res = solve_batch([KNOWN[n][0] for n in names], opts(1e-8))
    for n, r in zip(names, res):
        obj = KNOWN[n][1]
        assert r.status == SolveStatus.kOptimal, n
        assert abs(r.objective_value - obj) <= 1e-7 * (1 + abs(obj)), n


def test_batch_refines_to_1e8():
    models = [random_sparse_lp(300, 900, 4, seed=s) for s in (0, 1)] + [rolling_horizon_lp(24, 5, seed=2)]
    res = solve_batch(models, opts(1e-8, 400000))
    for model, r in zip(models, res):
        assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
        check(model, r, 1e-8)


def test_batch_early_answers_and_mixed_sense():
    empty = ModelIR([], [0, 0], [], [], [1.0], [2.0], [], [], 0, 4.5)      # one row, no variables
    bad = ModelIR([np.nan, 1.0], [0, 2], [0, 1], [1.0, 1.0], [1.0], [1.0], [0, 0], [10, 10], 0, 0.0)
    wyndor = KNOWN["wyndor"][0]                                          # maximisation
    res = solve_batch([empty, wyndor, bad], opts(1e-6))
    assert res[0].status == SolveStatus.kOptimal and res[0].objective_value == 4.5
    assert res[0].iterations == 0 and list(res[0].row_activity) == [0.0]
    assert res[1].status == SolveStatus.kOptimal
    assert res[1].objective_value == pytest.approx(36.0, rel=1e-5)
    assert res[2].status == SolveStatus.kNumericalFailure


def test_batch_is_deterministic():
    models = rolling_horizon_batch(16, seed=4, T_range=(24, 48), P_range=(5, 10))
    a = solve_batch(models, opts(1e-6))
    b = solve_batch(models, opts(1e-6))
    for ra, rb in zip(a, b):
        assert ra.iterations == rb.iterations
        assert np.array_equal(ra.x, rb.x) and np.array_equal(ra.y, rb.y)


def test_rolling_horizon_batch_certified():
    # big enough that the operand is rebuilt from the unconverged LPs on the way
    models = rolling_horizon_batch(48, seed=1, T_range=(24, 120), P_range=(5, 20))
    res = solve_batch(models, opts(1e-6))
    assert res[0].compactions >= 1
    for model, r in zip(models, res):
        assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
        check(model, r, 1e-6)
        cert = oracle.certificate(model, r.x)
        b = np.concatenate([model.row_lower[model.row_lower > -1e29], model.row_upper[model.row_upper < 1e29]])
        assert cert["primal_residual"] <= 1e-6 * (1 + np.linalg.norm(b))
