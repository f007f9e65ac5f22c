"""Batches of independent LPs over several GPUs: one process per GPU.

The LPs of a batch share nothing, so they shard by LP with no collective on
the data path: every rank takes a share chosen by a deterministic greedy
balance of the non-zeros (the per-iteration cost of a packed batch follows its
non-zeros), solves it with the batched PDHG on its own GPU, and the answers
are gathered once at the end.  ``torch.distributed`` is the plumbing (NCCL
between GPUs, gloo in the CPU tests); the solve itself never touches it.
"""
from __future__ import annotations

import numpy as np

from .pdhg import ModelIR, PdhgOptions, SolveResult, solve_batch


def shard_plan(nnz: list[int], world: int) -> list[list[int]]:
    """Greedy balance: LPs in decreasing order of non-zeros, each to the rank
    with the fewest non-zeros so far (ties to the lower rank).  Returns the LP
    indices of every rank, each list in increasing order; deterministic, so
    every rank computes the same plan."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    plan: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(nnz)), key=lambda k: (-int(nnz[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        plan[r].append(i)
        load[r] += int(nnz[i]) + 1          # +1: an LP without non-zeros still costs a little
    return [sorted(p) for p in plan]


def solve_batch_sharded(models: list[ModelIR], options: PdhgOptions | None = None, group=None,
                        gather: bool = True) -> list[SolveResult | None]:
    """Solves ``models`` over the ranks of ``group`` (torch.distributed; every
    rank passes the same list).  Rank r solves ``shard_plan(...)[r]`` on its
    device (``options.device``).  With ``gather`` every rank returns all
    results in the original order; without, the other ranks' slots are None."""
    import torch.distributed as dist

    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    plan = shard_plan([m.nnz() for m in models], world)
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
