"""Branch-and-bound node relaxations as one batch.

The reference's branch-and-bound (src/mip/branch_and_bound.cpp:39-65) solves
each node's LP relaxation — the model with the node's variable bounds — with
the dual simplex, warm-started from the parent's basis.  Here the relaxations
of many open nodes are packed into one batched PDHG solve, each warm-started
from its parent's primal-dual point (clamped into the node's bounds).
"""
from __future__ import annotations

import math

import numpy as np

from .gnn import WarmStart
from .pdhg import ModelIR, PdhgOptions, SolveResult, solve_batch


def node_relaxation(model: ModelIR, var_lower, var_upper) -> ModelIR:
    """The LP relaxation of a node: ``model`` with the node's variable bounds."""
    lo = np.asarray(var_lower, np.float64)
    hi = np.asarray(var_upper, np.float64)
    if lo.shape != (model.numVars(),) or hi.shape != (model.numVars(),):
        raise ValueError("node bounds must have one entry per variable")
    return ModelIR(model.obj_coeffs, model.row_ptr, model.col_idx, model.values, model.row_lower,
                   model.row_upper, lo, hi, model.obj_sense, model.obj_offset)


def branch(var_lower, var_upper, j: int, value: float):
    """The two children of branching on variable j at a fractional ``value``
    (BranchDirection::kDown: x_j <= floor(value); kUp: x_j >= ceil(value)),
    as (lower, upper) bound pairs."""
    lo = np.asarray(var_lower, np.float64)
    hi = np.asarray(var_upper, np.float64)
    down_hi = hi.copy()
    down_hi[j] = min(hi[j], math.floor(value))
    up_lo = lo.copy()
    up_lo[j] = max(lo[j], math.ceil(value))
    return (lo.copy(), down_hi), (up_lo, hi.copy())


def solve_node_relaxations(model: ModelIR, bounds: list[tuple], options: PdhgOptions | None = None,
                           parents: list[SolveResult | None] | None = None) -> list[SolveResult]:
    """Solves the relaxations of the nodes ``bounds[k] = (var_lower, var_upper)``
    as one batch; ``parents[k]`` (optional) is the solved parent whose point
    warm-starts node k."""
    models = [node_relaxation(model, lo, hi) for lo, hi in bounds]
    warm = None
    if parents is not None:
        if len(parents) != len(bounds):
            raise ValueError("one parent (or None) per node")
        warm = []
        for (lo, hi), p in zip(bounds, parents):
            if p is None:
                warm.append(None)
                continue
            x = np.clip(np.asarray(p.x, np.float64), lo, hi)
            warm.append(WarmStart(x, np.asarray(p.y, np.float64), 0.0))
    return solve_batch(models, options, warm=warm)
