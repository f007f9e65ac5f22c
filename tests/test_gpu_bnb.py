"""GPU tests of batched branch-and-bound node relaxations (pramaan_b200/bnb.py).

Checker: the reference's own RevisedSimplex (oracle/_ref) on every node LP;
the objectives agree to the tolerance of the FP64-refined PDHG.
"""
import numpy as np
import pytest

import oracle
from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus
from pramaan_b200.bnb import branch, node_relaxation, solve_node_relaxations
from pramaan_b200.generators import random_sparse_lp
from pramaan_b200.pdhg import ALGO_HALPERN

pytestmark = pytest.mark.gpu


def opts(tol=1e-8):
    return PdhgOptions(tolerance=tol, max_iterations=400000, check_frequency=64, algorithm=ALGO_HALPERN)


def test_children_of_the_root_match_the_cpu_simplex_and_warm_starts_help():
    if oracle.ref_cpu() is None:
        pytest.skip("oracle/_ref not built")
    md = random_sparse_lp(40, 120, 4, seed=5)
    root = PdhgSolver(opts()).solve(md)
    assert root.status == SolveStatus.kOptimal
    frac = [j for j in np.argsort(-np.abs(root.x - np.round(root.x)))[:6]
            if abs(root.x[j] - round(root.x[j])) > 1e-3]
    assert len(frac) >= 3
    bounds = []
    for j in frac:
        down, up = branch(md.var_lower, md.var_upper, int(j), float(root.x[j]))
        bounds += [down, up]
    cold = solve_node_relaxations(md, bounds, opts())
    warm = solve_node_relaxations(md, bounds, opts(), parents=[root] * len(bounds))
    for (lo, hi), c, w in zip(bounds, cold, warm):
        ref = oracle.ref_solve("simplex", node_relaxation(md, lo, hi), max_iterations=200000, tolerance=1e-9)
        assert ref["status"] == 0
        for r in (c, w):
            assert r.status == SolveStatus.kOptimal
            assert r.objective_value == pytest.approx(ref["objective_value"], rel=1e-6, abs=1e-6)
            assert np.all(r.x >= lo - 1e-7) and np.all(r.x <= hi + 1e-7)
    assert sum(r.iterations for r in warm) < sum(r.iterations for r in cold)


def test_branch_bounds():
    lo, hi = np.zeros(3), np.array([5.0, 1e30, 2.0])
    (dl, dh), (ul, uh) = branch(lo, hi, 1, 2.4)
    assert dh[1] == 2.0 and dl[1] == 0.0 and ul[1] == 3.0 and uh[1] == 1e30
    assert list(dh[[0, 2]]) == [5.0, 2.0] and list(ul[[0, 2]]) == [0.0, 0.0]
