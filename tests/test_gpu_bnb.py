"""GPU tests of batched branch-and-bound node relaxations (pramaan_b200/bnb.py).

Checker: the reference's own RevisedSimplex (oracle/_ref) on every node LP;
the objectives agree to the tolerance of the FP64-refined PDHG.
"""
import numpy as np
import pytest

import oracle
from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus
from pramaan_b200.bnb import branch, node_relaxation, solve_node_relaxations
from pramaan_b200.generators import rolling_horizon_lp
from pramaan_b200.pdhg import ALGO_HALPERN

pytestmark = pytest.mark.gpu


def opts(tol=1e-8, it=400000):
    return PdhgOptions(tolerance=tol, max_iterations=it, check_frequency=64, algorithm=ALGO_HALPERN)


def test_children_of_the_root_match_the_cpu_simplex_and_warm_starts_help():
    """Branching on fractional production quantities of a production-planning
    LP (backlog keeps the children feasible); a child the reference simplex
    finds infeasible must not come back optimal (PDHG stops at its limit)."""
    if oracle.ref_cpu() is None:
        pytest.skip("oracle/_ref not built")
    md = rolling_horizon_lp(12, 3, seed=5)
    root = PdhgSolver(opts()).solve(md)
    assert root.status == SolveStatus.kOptimal
    PT = md.numVars() // 3
    frac = [j for j in np.argsort(-np.abs(root.x[:PT] - np.round(root.x[:PT])))[:6]
            if abs(root.x[j] - round(root.x[j])) > 1e-3]
    assert len(frac) >= 3
    bounds = []
    for j in frac:
        down, up = branch(md.var_lower, md.var_upper, int(j), float(root.x[j]))
        bounds += [down, up]
    cold = solve_node_relaxations(md, bounds, opts(it=100000))
    warm = solve_node_relaxations(md, bounds, opts(it=100000), parents=[root] * len(bounds))
    feasible = 0
    for (lo, hi), c, w in zip(bounds, cold, warm):
        ref = oracle.ref_solve("simplex", node_relaxation(md, lo, hi), max_iterations=200000, tolerance=1e-9)
        if ref["status"] != 0:
            assert c.status != SolveStatus.kOptimal and w.status != SolveStatus.kOptimal
            continue
        feasible += 1
        for r in (c, w):
            assert r.status == SolveStatus.kOptimal
            assert r.objective_value == pytest.approx(ref["objective_value"], rel=1e-6, abs=1e-6)
            assert np.all(r.x >= lo - 1e-7) and np.all(r.x <= hi + 1e-7)
    assert feasible >= 4
    assert sum(r.iterations for r in warm) < sum(r.iterations for r in cold)


def test_branch_bounds():
    lo, hi = np.zeros(3), np.array([5.0, 1e30, 2.0])
    (dl, dh), (ul, uh) = branch(lo, hi, 1, 2.4)
    assert dh[1] == 2.0 and dl[1] == 0.0 and ul[1] == 3.0 and uh[1] == 1e30
    assert list(dh[[0, 2]]) == [5.0, 2.0] and list(ul[[0, 2]]) == [0.0, 0.0]
