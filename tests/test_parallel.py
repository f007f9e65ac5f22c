"""CPU tests of the multi-GPU sharding of LP batches (pramaan_b200/parallel.py).

The shard plan is host logic; the gather runs over torch.distributed with the
gloo backend on two CPU processes.  The per-rank solve is replaced by a fake
that records which LPs it received (no GPU here); on a GPU box the same code
runs the batched PDHG per rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from pramaan_b200 import parallel
from pramaan_b200.generators import rolling_horizon_batch


def test_shard_plan_covers_every_lp_once_and_balances_nonzeros():
    rng = np.random.default_rng(0)
    nnz = list(rng.integers(0, 100000, size=97))
    for world in (1, 2, 3, 8):
        plan = parallel.shard_plan(nnz, world)
        assert sorted(i for p in plan for i in p) == list(range(97))
        loads = [sum(nnz[i] + 1 for i in p) for p in plan]
        assert max(loads) - min(loads) <= max(nnz) + 1
        assert plan == parallel.shard_plan(nnz, world)          # deterministic
        assert all(p == sorted(p) for p in plan)
    assert parallel.shard_plan([], 4) == [[], [], [], []]
    assert parallel.shard_plan([5, 5, 5], 4)[3] == []
    with pytest.raises(ValueError):
        parallel.shard_plan([1], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    from pramaan_b200.pdhg import SolveResult, SolveStatus

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    models = rolling_horizon_batch(9, seed=3, T_range=(5, 12), P_range=(2, 4))
    seen = []

    def fake_solve(ms, options=None):
        res = []
        for md in ms:
            seen.append(md.numVars())
            r = SolveResult()
            r.status = SolveStatus.kOptimal
            r.x = np.full(md.numVars(), float(rank))
            r.y = np.zeros(md.numRows())
            r.row_activity = np.zeros(md.numRows())
            r.objective_value = float(md.nnz())
            res.append(r)
        return res

    parallel.solve_batch = fake_solve
    res = parallel.solve_batch_sharded(models, None)
    plan = parallel.shard_plan([m.nnz() for m in models], world)
    out.put((rank, seen, [(r.objective_value, float(r.x[0]), int(r.status)) for r in res],
             [m.nnz() for m in models], plan))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_solve_their_shards_and_gather_everything():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, seen, res, nnz, plan in got:
        # every rank solved exactly its planned LPs ...
        assert len(seen) == len(plan[rank])
        # ... and holds all answers, each from the rank that owns the LP
        assert [o for o, _, _ in res] == [float(v) for v in nnz]
        owner = {i: r for r, p in enumerate(plan) for i in p}
        assert [x for _, x, _ in res] == [float(owner[i]) for i in range(len(nnz))]
        assert all(s == 0 for _, _, s in res)


def test_shard_plan_with_iterations_equal_iterations_same_plan():
    rng = np.random.default_rng(1)
    nnz = list(rng.integers(0, 100000, size=61))
    for world in (1, 2, 3, 8):
        assert parallel.shard_plan(nnz, world, [5000.0] * 61) == parallel.shard_plan(nnz, world)


def test_shard_plan_with_iterations_balances_the_slow_lps():
    # rolling-horizon-like: many LPs of ~20-90 k iterations, a few of ~300 k, non-zeros
    # unrelated to the iterations; the iteration-aware plan's modelled makespan is never
    # worse than the non-zeros-only plan's, and better here
    rng = np.random.default_rng(2)
    n = 128
    nnz = list(rng.integers(2_000, 90_000, size=n))
    iters = list(rng.integers(20_000, 90_000, size=n).astype(float))
    for k in rng.choice(n, 4, replace=False):
        iters[k] = 300_000.0
    for world in (2, 4, 8):
        plan_it = parallel.shard_plan(nnz, world, iters)
        plan_nz = parallel.shard_plan(nnz, world)
        assert sorted(i for p in plan_it for i in p) == list(range(n))
        assert plan_it == parallel.shard_plan(nnz, world, iters)     # deterministic
        span_it = max(parallel.rank_seconds(nnz, iters, p) for p in plan_it)
        span_nz = max(parallel.rank_seconds(nnz, iters, p) for p in plan_nz)
        assert span_it <= span_nz * (1 + 1e-12)
    assert span_it < span_nz
    with pytest.raises(ValueError):
        parallel.shard_plan([1, 2], 2, [1.0])
    with pytest.raises(ValueError):
        parallel.shard_plan([1, 2], 2, [1.0, -1.0])
