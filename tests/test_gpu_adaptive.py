"""GPU tests of the adaptive restarted PDHG mode (PRAMAAN_ALGO_ADAPTIVE with
relative-KKT termination).

The mode has no reference counterpart; it is judged by the oracle's FP64
relative-KKT restatement (oracle/pdhg_oracle.c orc_rel_kkt, PDLP definitions)
on the returned (x, y), by the reference's known optima, and by the
reference's own simplex where that finishes.  Tolerances:
  * the reported relative KKT components equal the oracle's recomputation
    on the returned iterate within 1e-6 relative (both FP64; the device sums
    in another order);
  * at tolerance t the oracle's relative KKT is <= t (primal, dual, gap);
    FP32 iterates resolve about 1e-7, so these FP32-only solves ask for
    1e-6 at most (1e-8 is the FP64 refinement's job);
  * objectives agree with known optima / simplex within 1e-4 * (1 + |obj|).
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN, mps_model, primal_violation
from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus
from pramaan_b200.generators import ill_conditioned_lp, random_sparse_lp, zipf_lp
from pramaan_b200.pdhg import ALGO_ADAPTIVE, TERM_RELATIVE_KKT

pytestmark = pytest.mark.gpu


def adaptive(tol=1e-6, max_it=200000, cf=64):
    return PdhgSolver(PdhgOptions(tolerance=tol, max_iterations=max_it, check_frequency=cf,
                                  algorithm=ALGO_ADAPTIVE, termination=TERM_RELATIVE_KKT))


def check_kkt(model, r, tol):
    k = oracle.rel_kkt(model, r.x, r.y)
    assert k["primal"] <= tol * 1.0001 and k["dual"] <= tol * 1.0001 and k["gap"] <= tol * 1.0001, k
    for mine, theirs in ((r.rel_primal, k["primal"]), (r.rel_dual, k["dual"]), (r.rel_gap, k["gap"])):
        assert mine == pytest.approx(theirs, rel=1e-6, abs=1e-12)
    return k


@pytest.mark.parametrize("name", sorted(KNOWN))
def test_adaptive_known_answers(name):
    model, obj, feas = KNOWN[name]
    r = adaptive(1e-6).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.status, r.iterations)
    assert abs(r.objective_value - obj) <= 1e-4 * (1 + abs(obj))
    if feas:
        assert primal_violation(model, r.x) <= 1e-5


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_adaptive_random_lp_meets_relative_kkt(seed):
    model = random_sparse_lp(300, 900, 4, seed=seed)
    r = adaptive(1e-6).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-6)


def test_adaptive_matches_reference_simplex():
    model = random_sparse_lp(40, 120, 4, seed=3)
    cpu = oracle.ref_solve("simplex", model, max_iterations=100000) if oracle.ref_cpu() else None
    r = adaptive(1e-6).solve(model)
    assert r.status == SolveStatus.kOptimal
    check_kkt(model, r, 1e-6)
    if cpu is not None and cpu["status"] == 0:
        assert r.objective_value == pytest.approx(cpu["objective_value"], rel=1e-4, abs=1e-4)


def test_adaptive_afiro():
    model = mps_model("afiro")
    if model is None:
        pytest.skip("oracle/_ref not built")
    r = adaptive(1e-6).solve(model)
    assert r.status == SolveStatus.kOptimal
    assert r.objective_value == pytest.approx(-464.75314286, rel=1e-5)
    check_kkt(model, r, 1e-6)


def test_adaptive_converges_faster_than_reference_iteration():
    model = random_sparse_lp(200, 600, 4, seed=5)
    ref = PdhgSolver(PdhgOptions(tolerance=1e-4, max_iterations=100000)).solve(model)
    ada = adaptive(1e-4).solve(model)
    assert ada.status == SolveStatus.kOptimal
    if ref.status == SolveStatus.kOptimal:
        assert abs(ada.objective_value - ref.objective_value) <= 1e-3 * (1 + abs(ref.objective_value))
    assert ada.iterations < ref.iterations


def test_adaptive_power_law_and_ill_conditioned():
    for model, tol in ((zipf_lp(3000, 9000, cap=500, seed=2), 1e-5),
                       (ill_conditioned_lp(2000, 5000, 8, seed=1, scale_exp=2.0), 1e-4)):
        r = adaptive(tol, max_it=300000).solve(model)
        assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
        check_kkt(model, r, tol)


def test_adaptive_deterministic():
    model = random_sparse_lp(300, 900, 4, seed=9)
    a = adaptive(1e-6).solve(model)
    b = adaptive(1e-6).solve(model)
    assert a.iterations == b.iterations and np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


# ---- FP64 iterative refinement (refine_rounds > 0): 1e-8 relative KKT ----

def refined(tol_inner=1e-5, target=1e-8, rounds=8, max_it=200000):
    return PdhgSolver(PdhgOptions(tolerance=tol_inner, max_iterations=max_it, check_frequency=64,
                                  algorithm=ALGO_ADAPTIVE, termination=TERM_RELATIVE_KKT,
                                  refine_rounds=rounds, refine_tolerance=target))


@pytest.mark.parametrize("name", ["multi", "wyndor", "bounded", "equality", "one_var"])
def test_refined_known_answers_reach_1e8(name):
    model, obj, _ = KNOWN[name]
    r = refined().solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)
    assert abs(r.objective_value - obj) <= 1e-8 * (1 + abs(obj))


@pytest.mark.parametrize("seed", [0, 1])
def test_refined_random_lp_reaches_1e8(seed):
    model = random_sparse_lp(300, 900, 4, seed=seed)
    r = refined().solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)


def test_refined_afiro_matches_simplex_to_1e8():
    model = mps_model("afiro")
    if model is None:
        pytest.skip("oracle/_ref not built")
    r = refined().solve(model)
    assert r.status == SolveStatus.kOptimal
    check_kkt(model, r, 1e-8)
    cpu = oracle.ref_solve("simplex", model)
    assert r.objective_value == pytest.approx(cpu["objective_value"], rel=1e-8)


def test_refined_ill_conditioned():
    model = ill_conditioned_lp(2000, 5000, 8, seed=2, scale_exp=3.0)
    r = refined(tol_inner=1e-4, rounds=12, max_it=400000).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)
