"""Batches of independent LPs over several GPUs: one process per GPU.

The LPs of a batch share nothing, so they shard by LP with no collective on
the data path: every rank takes a share chosen by a deterministic greedy
balance of the non-zeros (the per-iteration cost of a packed batch follows its
non-zeros), or, when the caller knows how many iterations each LP will need
(a rolling-horizon stream does, from the previous window), of a time model that
also charges the slowest LP's iterations; it solves its share with the batched
PDHG on its own GPU, and the answers are gathered once at the end.  ``torch.distributed`` is the plumbing (NCCL
between GPUs, gloo in the CPU tests); the solve itself never touches it.
"""
from __future__ import annotations

import numpy as np

from .pdhg import ModelIR, PdhgOptions, SolveResult, solve_batch


# Time model of one rank's packed batch (B200, restarted Halpern PDHG on the
# 512-LP rolling-horizon batch): while many LPs iterate, an iteration costs
# its live non-zeros times NNZ_ITER_SECONDS (176 us per iteration with all
# 15,951,002 non-zeros live); an iteration never costs less than
# ITER_LATENCY_SECONDS (13 us: the batch's last LP alone on the per-LP cluster
# kernel).  So a rank needs about
#   NNZ_ITER_SECONDS * sum_i (nnz_i + 1) * iters_i + ITER_LATENCY_SECONDS * max_i iters_i,
# and the LP that needs the most iterations sets the second term: with the
# non-zeros alone, a rank that draws two of the slowest LPs and its share of
# the others finishes last.
NNZ_ITER_SECONDS = 176e-6 / 15_951_002
ITER_LATENCY_SECONDS = 13e-6


def rank_seconds(nnz: list[int], iterations: list[float], lps: list[int]) -> float:
    """The time model above for the LPs `lps` of one rank."""
    if not lps:
        return 0.0
    bulk = sum((int(nnz[i]) + 1) * float(iterations[i]) for i in lps)
    return NNZ_ITER_SECONDS * bulk + ITER_LATENCY_SECONDS * max(float(iterations[i]) for i in lps)


def shard_plan(nnz: list[int], world: int, iterations: list[float] | None = None) -> list[list[int]]:
    """Greedy balance of the LPs over `world` ranks.  Returns the LP indices of
    every rank, each list in increasing order; deterministic, so every rank
    computes the same plan.

    Without `iterations`: LPs in decreasing order of non-zeros, each to the
    rank with the fewest non-zeros so far (ties to the lower rank).

    With `iterations` (expected iterations per LP, e.g. each LP's count in the
    previous window of a rolling-horizon stream): LPs in decreasing order of
    expected iterations (then non-zeros), each to the rank whose modelled time
    (rank_seconds) after taking it is smallest (ties to the lower rank).  With
    equal iterations this is the same plan as the non-zeros alone."""
    if world < 1:
        raise ValueError("world must be >= 1")
    plan: list[list[int]] = [[] for _ in range(world)]
    if iterations is None:
        load = [0] * world
        for i in sorted(range(len(nnz)), key=lambda k: (-int(nnz[k]), k)):
            r = min(range(world), key=lambda q: (load[q], q))
            plan[r].append(i)
            load[r] += int(nnz[i]) + 1          # +1: an LP without non-zeros still costs a little
        return [sorted(p) for p in plan]
    if len(iterations) != len(nnz):
        raise ValueError("iterations must give one count per LP")
    if any(not (float(t) >= 0.0) for t in iterations):
        raise ValueError("expected iterations must be non-negative numbers")
    bulk = [0.0] * world
    most = [0.0] * world

    def after(q: int, i: int) -> float:
        it = float(iterations[i])
        return (NNZ_ITER_SECONDS * (bulk[q] + (int(nnz[i]) + 1) * it)
                + ITER_LATENCY_SECONDS * max(most[q], it))

    for i in sorted(range(len(nnz)), key=lambda k: (-float(iterations[k]), -int(nnz[k]), k)):
        r = min(range(world), key=lambda q: (after(q, i), q))
        plan[r].append(i)
        bulk[r] += (int(nnz[i]) + 1) * float(iterations[i])
        most[r] = max(most[r], float(iterations[i]))
    return [sorted(p) for p in plan]


def solve_batch_sharded(models: list[ModelIR], options: PdhgOptions | None = None, group=None,
                        gather: bool = True, iterations: list[float] | None = None) -> list[SolveResult | None]:
    """Solves ``models`` over the ranks of ``group`` (torch.distributed; every
    rank passes the same list).  Rank r solves ``shard_plan(...)[r]`` on its
    device (``options.device``), the plan balanced on ``iterations`` too when
    given (every rank must pass the same).  With ``gather`` every rank returns
    all results in the original order; without, the other ranks' slots are
    None."""
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    plan = shard_plan([m.nnz() for m in models], world, iterations)
    mine = plan[rank]
    res = solve_batch([models[i] for i in mine], options) if mine else []
    out: list[SolveResult | None] = [None] * len(models)
    for i, r in zip(mine, res):
        out[i] = r
    if gather and world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, [(i, _pack(r)) for i, r in zip(mine, res)], group=group)
        for part in parts:
            for i, packed in part:
                out[i] = _unpack(packed)
    return out


def _pack(r: SolveResult) -> dict:
    d = dict(r.__dict__)
    d["status"] = int(r.status)
    return d


def _unpack(d: dict) -> SolveResult:
    from .pdhg import SolveStatus

    r = SolveResult()
    for k, v in d.items():
        setattr(r, k, v)
    r.status = SolveStatus(d["status"])
    for k in ("x", "y", "row_activity"):
        setattr(r, k, np.asarray(getattr(r, k)))
    return r
