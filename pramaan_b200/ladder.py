"""Precision ladder: the reference's GPU-then-CPU controller with a GPU FP64 rung.

Mirrors pramaan::PrecisionLadder (include/pramaan/gpu/precision_ladder.hpp,
src/gpu/precision_ladder.cpp:55-181): rung 1 is the reference FP32 PDHG,
accepted iff it is optimal and both reference residuals are within
``residual_threshold``.  Before escalating, rung 2 (``refine=True``) runs the
adaptive PDHG with FP64 iterative refinement on the GPU and applies the same
gate.  Rung 3 is the caller's CPU FP64 solver (the reference runs its
RevisedSimplex with the GPU x as primal start hint): pass it as
``cpu_solver(model, hint_x) -> SolveResult``; without one, an escalated result
carries the best GPU point and ``final_result`` is None.
"""
from __future__ import annotations

import ctypes as C
import enum
import time
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .pdhg import ModelIR, SolveResult, SolveStatus, _ptr


class Stage(enum.IntEnum):
    kGpuFp32 = 0
    kGpuFp64Refined = 1
    kCpuFp64Polish = 2


class EscalationReason(enum.IntEnum):
    """PrecisionLadderResult::EscalationReason (include/pramaan/gpu/precision_ladder.hpp)."""
    kNone = 0
    kHighPrimalResidual = 1
    kHighDualResidual = 2
    kGpuIterationLimit = 3
    kGpuNumericalFailure = 4
    kGpuNotOptimal = 5
    kGpuDisabled = 6


@dataclass
class LadderOptions:
    residual_threshold: float = 1e-6
    gpu_max_iterations: int = 100000
    gpu_check_frequency: int = 100
    gpu_tolerance: float = 1e-6
    refine: bool = True
    refine_max_iterations: int = 400000
    refine_tolerance: float = 1e-9
    device: int = 0


@dataclass
class PrecisionLadderResult:
    final_result: SolveResult | None = None
    stage: Stage = Stage.kCpuFp64Polish
    escalated: bool = False
    escalation_reason: EscalationReason = EscalationReason.kNone
    refine_escalation_reason: EscalationReason = EscalationReason.kNone
    gpu_status: SolveStatus = SolveStatus.kIterationLimit
    gpu_primal_residual: float = float("inf")
    gpu_dual_residual: float = float("inf")
    gpu_objective: float = 0.0
    gpu_iterations: int = 0
    gpu_elapsed_ms: float = 0.0
    refine_status: SolveStatus = SolveStatus.kIterationLimit
    refine_iterations: int = 0
    refine_primal_residual: float = float("inf")
    refine_dual_residual: float = float("inf")
    refine_elapsed_ms: float = 0.0
    cpu_elapsed_ms: float = 0.0
    total_elapsed_ms: float = 0.0
    gpu_x: np.ndarray = field(default_factory=lambda: np.zeros(0))
    gpu_y: np.ndarray = field(default_factory=lambda: np.zeros(0))
    rel_primal: float = float("nan")
    rel_dual: float = float("nan")
    rel_gap: float = float("nan")


class PrecisionLadder:
    def __init__(self, options: LadderOptions | None = None, cpu_solver=None):
        self.options = options or LadderOptions()
        self.cpu_solver = cpu_solver

    def solve(self, model: ModelIR) -> PrecisionLadderResult:
        o = L.CLadderOptions()
        L.lib().pramaan_ladder_default_options(C.byref(o))
        for f in ("residual_threshold", "gpu_max_iterations", "gpu_check_frequency", "gpu_tolerance",
                  "refine_max_iterations", "refine_tolerance", "device"):
            setattr(o, f, getattr(self.options, f))
        o.refine = int(bool(self.options.refine))
        n, m = model.numVars(), model.numRows()
        x, y, act = np.zeros(n), np.zeros(m), np.zeros(m)
        r = L.CLadderResult()
        r.x, r.y, r.row_activity = _ptr(x), _ptr(y), _ptr(act)
        lp = model.c_struct()
        t0 = time.perf_counter()
        L.check(L.lib().pramaan_ladder_solve(C.byref(lp), C.byref(o), C.byref(r)))
        out = PrecisionLadderResult(
            stage=Stage(r.stage), escalation_reason=EscalationReason(r.escalation_reason),
            refine_escalation_reason=EscalationReason(r.refine_escalation_reason),
            gpu_status=SolveStatus(r.gpu_status), gpu_primal_residual=r.gpu_primal_residual,
            gpu_dual_residual=r.gpu_dual_residual, gpu_objective=r.gpu_objective,
            gpu_iterations=r.gpu_iterations, gpu_elapsed_ms=r.gpu_elapsed_ms,
            refine_status=SolveStatus(r.refine_status), refine_iterations=r.refine_iterations,
            refine_primal_residual=r.refine_primal_residual, refine_dual_residual=r.refine_dual_residual,
            refine_elapsed_ms=r.refine_elapsed_ms, gpu_x=x, gpu_y=y,
            rel_primal=r.rel_primal, rel_dual=r.rel_dual, rel_gap=r.rel_gap)
        out.escalated = out.stage == Stage.kCpuFp64Polish
        if not out.escalated:
            fr = SolveResult()
            fr.status = SolveStatus.kOptimal
            fr.x, fr.y, fr.row_activity = x, y, act
            fr.objective_value = r.objective_value
            if out.stage == Stage.kGpuFp32:
                fr.iterations, fr.primal_residual, fr.dual_residual = (r.gpu_iterations, r.gpu_primal_residual,
                                                                       r.gpu_dual_residual)
            else:
                fr.iterations, fr.primal_residual, fr.dual_residual = (r.refine_iterations, r.refine_primal_residual,
                                                                       r.refine_dual_residual)
            fr.rel_primal, fr.rel_dual, fr.rel_gap = r.rel_primal, r.rel_dual, r.rel_gap
            out.final_result = fr
        elif self.cpu_solver is not None:
            t1 = time.perf_counter()
            out.final_result = self.cpu_solver(model, x)
            out.cpu_elapsed_ms = (time.perf_counter() - t1) * 1e3
        out.total_elapsed_ms = (time.perf_counter() - t0) * 1e3
        return out
