"""Time one solve of a generated LP.

Usage:
    python -m pramaan_b200.solve_bench [--lp rolling|random|ill|zipf] [--size A B]
        [--algorithm reference|adaptive|halpern] [--tol 1e-6] [--max-iterations N]
        [--batch K] [--seed 0] [--persistent -1|0|1]

`--lp rolling --size T P` is rolling_horizon_lp(T, P); `random --size m n` is
random_sparse_lp(m, n, 4); `ill --size m n` is ill_conditioned_lp(m, n, 8);
`zipf --size m n` is zipf_lp(m, n).  `--batch K` solves K copies with
different seeds as one batch.  Prints one JSON line: iterations, status,
seconds, iterations per second and microseconds per iteration (wall time of
the whole call, upload and result included).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

if __package__ in (None, ""):
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

from pramaan_b200 import PdhgOptions, PdhgSolver, solve_batch  # noqa: E402
from pramaan_b200 import generators as gen  # noqa: E402
from pramaan_b200.pdhg import ALGO_ADAPTIVE, ALGO_HALPERN, ALGO_REFERENCE  # noqa: E402


def make(kind: str, a: int, b: int, seed: int):
    if kind == "rolling":
        return gen.rolling_horizon_lp(a, b, seed=seed)
    if kind == "random":
        return gen.random_sparse_lp(a, b, 4, seed=seed)
    if kind == "ill":
        return gen.ill_conditioned_lp(a, b, 8, seed=seed)
    if kind == "zipf":
        return gen.zipf_lp(a, b, seed=seed)
    raise ValueError(kind)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lp", default="rolling", choices=["rolling", "random", "ill", "zipf"])
    ap.add_argument("--size", type=int, nargs=2, default=(300, 45))
    ap.add_argument("--algorithm", default="halpern", choices=["reference", "adaptive", "halpern"])
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--max-iterations", type=int, default=300000)
    ap.add_argument("--check-frequency", type=int, default=64)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--persistent", type=int, default=0, choices=[-1, 0, 1])
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    algo = {"reference": ALGO_REFERENCE, "adaptive": ALGO_ADAPTIVE, "halpern": ALGO_HALPERN}[a.algorithm]
    o = PdhgOptions(tolerance=a.tol, max_iterations=a.max_iterations, check_frequency=a.check_frequency,
                    algorithm=algo, device=a.device, persistent=a.persistent)
    if a.batch:
        models = [make(a.lp, *a.size, seed=a.seed + k) for k in range(a.batch)]
        solve_batch(models[:1], o)                 # warm-up (module load)
        t0 = time.perf_counter()
        res = solve_batch(models, o)
        dt = time.perf_counter() - t0
        its = max(r.iterations for r in res)
        status = [r.status.name for r in res]
    else:
        md = make(a.lp, *a.size, seed=a.seed)
        solver = PdhgSolver(o)
        solver.solve(make(a.lp, 8, 2, seed=1) if a.lp == "rolling" else md)   # warm-up
        t0 = time.perf_counter()
        r = solver.solve(md)
        dt = time.perf_counter() - t0
        its, status = r.iterations, r.status.name
    print(json.dumps({"lp": a.lp, "size": list(a.size), "batch": a.batch, "algorithm": a.algorithm,
                      "persistent": a.persistent,
                      "tol": a.tol, "iterations": its, "status": status, "seconds": dt,
                      "iterations_per_s": its / dt if dt > 0 else None,
                      "us_per_iteration": 1e6 * dt / its if its else None}))


if __name__ == "__main__":
    main()
