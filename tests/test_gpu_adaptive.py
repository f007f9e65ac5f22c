"""GPU tests of the adaptive restarted PDHG mode (PRAMAAN_ALGO_ADAPTIVE with
relative-KKT termination) and its FP64 iterative refinement.

The mode has no reference counterpart; it is judged by the oracle's FP64
relative-KKT restatement (oracle/pdhg_oracle.c orc_rel_kkt, PDLP definitions)
on the returned (x, y), by the reference's known optima, by the reference's
own simplex where that finishes, and by the numpy restatement of the method
(oracle/adaptive.py) for its preconditioned step size and primal weight.
Tolerances:
  * the reported relative KKT components equal the oracle's recomputation
    on the returned FP64 iterate within 1e-4 relative (both FP64 sums, in
    another order; the gap is a difference of near-equal objectives);
  * at tolerance t the oracle's relative KKT is <= t (primal, dual, gap);
  * with refinement (the default) t goes down to 1e-8; plain FP32 iterates
    (refine=False) resolve about 1e-6 and are asked for 1e-5;
  * objectives agree with known optima / simplex within 1e-4 * (1 + |obj|)
    at t = 1e-6 and 1e-8 * (1 + |obj|) at t = 1e-8;
  * step size eta and the initial primal weight match the numpy
    restatement within 1e-2 relative (FP32 scales, power iteration stopped
    at a 1e-4 relative change).
"""
import numpy as np
import pytest

import oracle
from oracle import adaptive as ada_oracle
from lp_cases import KNOWN, mps_model, primal_violation
from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus
from pramaan_b200.generators import ill_conditioned_lp, random_sparse_lp, zipf_lp
from pramaan_b200.pdhg import ALGO_ADAPTIVE

pytestmark = pytest.mark.gpu


def adaptive(tol=1e-6, max_it=200000, cf=64, refine=True):
    return PdhgSolver(PdhgOptions(tolerance=tol, max_iterations=max_it, check_frequency=cf,
                                  algorithm=ALGO_ADAPTIVE, refine=refine))


def check_kkt(model, r, tol):
    k = oracle.rel_kkt(model, r.x, r.y)
    assert k["primal"] <= tol * 1.0001 and k["dual"] <= tol * 1.0001 and k["gap"] <= tol * 1.0001, k
    for mine, theirs in ((r.rel_primal, k["primal"]), (r.rel_dual, k["dual"]), (r.rel_gap, k["gap"])):
        assert mine == pytest.approx(theirs, rel=1e-4, abs=1e-13)
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


# ---- FP64 iterative refinement: FP64 master + FP32 corrections -> 1e-8 ----

def test_plain_fp32_iterates_reach_1e5():
    model = random_sparse_lp(300, 900, 4, seed=0)
    r = adaptive(1e-5, refine=False).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-5)


def test_refinement_is_what_reaches_1e8():
    # Rounding this LP's exact optimum to FP32 leaves a relative gap of about
    # 2e-6, so plain FP32 iterates cannot meet 1e-8; the refined solve does.
    model = random_sparse_lp(300, 900, 4, seed=1)
    plain = adaptive(1e-8, max_it=30000, refine=False).solve(model)
    assert plain.status == SolveStatus.kIterationLimit
    assert max(plain.rel_primal, plain.rel_dual, plain.rel_gap) > 1e-7
    r = adaptive(1e-8, max_it=200000).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)


@pytest.mark.parametrize("name", ["multi", "wyndor", "bounded", "equality", "one_var"])
def test_refined_known_answers_reach_1e8(name):
    model, obj, _ = KNOWN[name]
    r = adaptive(1e-8).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)
    assert abs(r.objective_value - obj) <= 1e-7 * (1 + abs(obj))


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_refined_random_lp_reaches_1e8(seed):
    model = random_sparse_lp(300, 900, 4, seed=seed)
    r = adaptive(1e-8).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)


def test_refined_afiro_matches_simplex_to_1e8():
    model = mps_model("afiro")
    if model is None:
        pytest.skip("oracle/_ref not built")
    r = adaptive(1e-8, max_it=400000).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)
    cpu = oracle.ref_solve("simplex", model)
    assert r.objective_value == pytest.approx(cpu["objective_value"], rel=1e-7)


def test_refined_ill_conditioned():
    model = ill_conditioned_lp(2000, 5000, 8, seed=2, scale_exp=3.0)
    r = adaptive(1e-8, max_it=400000).solve(model)
    assert r.status == SolveStatus.kOptimal, (r.iterations, r.rel_primal, r.rel_dual, r.rel_gap)
    check_kkt(model, r, 1e-8)


# ---- the preconditioner against the numpy restatement ------------------------

@pytest.mark.parametrize("seed", [0, 3])
def test_step_size_and_initial_weight_match_restatement(seed):
    model = random_sparse_lp(200, 500, 5, seed=seed)
    r = adaptive(1e-6, max_it=0).solve(model)
    P = ada_oracle.problem(model)
    R, C, sigma, tau = ada_oracle.steps(P)
    eta = 0.99 / ada_oracle.op_norm(P, sigma, tau)
    omega = ada_oracle.initial_weight(P, R, C)
    assert r.step_size == pytest.approx(eta, rel=1e-2)
    assert r.primal_weight == pytest.approx(omega, rel=1e-2)
