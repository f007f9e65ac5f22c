"""GPU tests of the precision ladder (pramaan_ladder_solve).

Rung 1 is the reference's own gate (src/gpu/precision_ladder.cpp:91-121) on
the reference FP32 PDHG; rung 2 is the GPU FP64 refinement judged by the same
gate; rung 3 is the caller's CPU solver — here the reference's own
RevisedSimplex (oracle/_ref), as in the reference controller.  Acceptance is
checked independently with the oracle's FP64 certificate
(src/certificate/certificate.cpp:23-107).
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN
from pramaan_b200.generators import ill_conditioned_lp, random_sparse_lp
from pramaan_b200.ladder import EscalationReason, LadderOptions, PrecisionLadder, Stage

pytestmark = pytest.mark.gpu


def cpu_simplex(model, hint):
    """The reference's RevisedSimplex with the GPU x as start hint."""
    from pramaan_b200.pdhg import SolveResult, SolveStatus
    r = oracle.ref_solve("simplex", model, max_iterations=200000, tolerance=1e-9, hint=hint)
    out = SolveResult()
    out.status = SolveStatus(r["status"])
    out.x = r["x"]
    out.objective_value = r["objective_value"]
    return out


def test_loose_threshold_accepts_the_fp32_rung():
    wy, obj = KNOWN["wyndor"][0], KNOWN["wyndor"][1]
    r = PrecisionLadder(LadderOptions(residual_threshold=1e-3, gpu_tolerance=1e-4)).solve(wy)
    assert r.stage == Stage.kGpuFp32 and not r.escalated
    assert r.escalation_reason == EscalationReason.kNone
    assert r.gpu_primal_residual <= 1e-3 and r.gpu_dual_residual <= 1e-3
    assert r.final_result.objective_value == pytest.approx(obj, rel=1e-3)


@pytest.mark.parametrize("seed", [0, 1])
def test_strict_threshold_is_met_by_the_fp64_rung(seed):
    md = ill_conditioned_lp(300, 800, 4, seed=seed, scale_exp=1.5)
    T = 1e-7
    r = PrecisionLadder(LadderOptions(residual_threshold=T, refine_tolerance=1e-10)).solve(md)
    assert r.escalation_reason != EscalationReason.kNone        # FP32 alone does not meet T
    assert r.stage == Stage.kGpuFp64Refined, (r.refine_status, r.refine_primal_residual, r.refine_dual_residual)
    cert = oracle.certificate(md, r.final_result.x)
    assert max(cert["primal_residual"], cert["bound_violation"]) <= T
    kk = oracle.rel_kkt(md, r.final_result.x, r.final_result.y)
    assert max(kk["primal"], kk["dual"], kk["gap"]) <= 1e-10 * 1.0001


def test_escalation_hands_the_gpu_point_to_the_cpu_solver():
    if oracle.ref_cpu() is None:
        pytest.skip("oracle/_ref not built")
    md = random_sparse_lp(60, 180, 4, seed=3)
    # no refinement rung, unattainable threshold: the reference's behaviour
    r = PrecisionLadder(LadderOptions(residual_threshold=1e-14, refine=False), cpu_solver=cpu_simplex).solve(md)
    assert r.escalated and r.stage == Stage.kCpuFp64Polish
    assert r.escalation_reason in (EscalationReason.kHighPrimalResidual, EscalationReason.kHighDualResidual,
                                   EscalationReason.kGpuIterationLimit)
    assert r.refine_iterations == 0
    ref = oracle.ref_solve("simplex", md, max_iterations=200000, tolerance=1e-9)
    assert r.final_result.objective_value == pytest.approx(ref["objective_value"], rel=1e-9, abs=1e-9)
    assert len(r.gpu_x) == md.numVars() and np.isfinite(r.gpu_x).all()


def test_refined_rung_that_misses_the_threshold_still_escalates():
    md = random_sparse_lp(60, 180, 4, seed=4)
    r = PrecisionLadder(LadderOptions(residual_threshold=1e-30, refine_tolerance=1e-9)).solve(md)
    assert r.escalated and r.final_result is None
    assert r.refine_iterations > 0
    assert r.refine_escalation_reason != EscalationReason.kNone
    # the hint is the better GPU point: the refined one
    kk = oracle.rel_kkt(md, r.gpu_x, r.gpu_y)
    assert max(kk["primal"], kk["dual"], kk["gap"]) <= 1e-9 * 1.0001
