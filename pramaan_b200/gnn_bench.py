"""Throughput of the warm-start network on a batch of rolling-horizon LPs.

Usage:
    python -m pramaan_b200.gnn_bench [--lps 64] [--reps 5] [--seed 0]

Builds a batch with the batched benchmark's shapes (T ~ U{24..336},
P ~ U{5..50}), then times the forward pass (predict) and one training step
(forward + backward + Adam) over it.  Prints one JSON line with the graph
size, the times and the dense layers' algorithmic work: per layer and side
2 * rows * 128 * 64 FLOPs forward, twice that backward (input and weight
gradients), and 384 bytes per row forward (a 256-byte BF16 input row read,
a 128-byte output row written).
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

if __package__ in (None, ""):
    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))

from pramaan_b200.generators import rolling_horizon_batch  # noqa: E402
from pramaan_b200.gnn import WarmStart, WarmStartNet  # noqa: E402


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--lps", type=int, default=64)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    models = rolling_horizon_batch(a.lps, seed=a.seed)
    m = sum(md.numRows() for md in models)
    n = sum(md.numVars() for md in models)
    rng = np.random.default_rng(a.seed)
    targets = [WarmStart(rng.uniform(0, 10, md.numVars()), rng.normal(0, 1, md.numRows()), 1.0) for md in models]
    net = WarmStartNet(device=a.device, seed=0)
    t0 = time.perf_counter()
    g = net.graph(models, targets)
    t_graph = time.perf_counter() - t0
    net.predict(g)
    net.train_step(g, 1e-4)
    t0 = time.perf_counter()
    for _ in range(a.reps):
        net.predict(g)
    t_fwd = (time.perf_counter() - t0) / a.reps
    t0 = time.perf_counter()
    for _ in range(a.reps):
        net.train_step(g, 1e-4)
    t_step = (time.perf_counter() - t0) / a.reps
    layers = 3
    dense_fwd_flops = layers * 2 * 128 * 64 * (m + n)
    print(json.dumps({"lps": a.lps, "rows": m, "cols": n, "nodes": m + n,
                      "nnz": sum(md.nnz() for md in models), "graph_build_s": t_graph,
                      "forward_ms": t_fwd * 1e3, "train_step_ms": t_step * 1e3,
                      "dense_forward_flops": dense_fwd_flops, "dense_train_flops": 3 * dense_fwd_flops,
                      "dense_forward_bytes": layers * 384 * (m + n),
                      "nodes_per_s_forward": (m + n) / t_fwd, "nodes_per_s_train": (m + n) / t_step}))


if __name__ == "__main__":
    main()
