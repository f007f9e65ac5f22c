"""Train the warm-start network on solved rolling-horizon windows (GPU).

Usage:
    python -m pramaan_b200.train_warm_start [--streams S] [--windows W] [--epochs E]
        [--T 24 96] [--P 5 20] [--seed0 N] [--out PATH]

Generates S streams of W consecutive windows (rolling_horizon_stream: AR(1)
demand, the window shifting by one period), labels every window with the
batched restarted Halpern PDHG (1e-6 relative KKT by default, ``--tol``), builds each window's hint (the
previous window's solution shifted by one period; none for a stream's first
window) and fits the network with Adam on mini-batches of 16 hinted windows.
The labels are the PDHG's own solutions, so the network learns nothing the
solver did not produce.  Writes the parameters (a flat float32 vector) and
the training record to ``--out`` (.npz).
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

from pramaan_b200 import PdhgOptions, SolveStatus, solve_batch  # noqa: E402
from pramaan_b200.generators import rolling_horizon_shift, rolling_horizon_stream  # noqa: E402
from pramaan_b200.gnn import WarmStart, WarmStartNet, training_targets  # noqa: E402
from pramaan_b200.pdhg import ALGO_HALPERN  # noqa: E402

DEFAULT_OUT = Path(__file__).resolve().parent / "weights" / "warm_start_rolling_horizon.npz"


def stream_windows(seeds, windows, T_range, P_range):
    """(models, first-window flags) of several streams, stream after stream."""
    ms, first = [], []
    for s in seeds:
        ms += rolling_horizon_stream(windows, seed=int(s), T_range=T_range, P_range=P_range)
        first += [True] + [False] * (windows - 1)
    return ms, first


def shifted_hints(models, first, results):
    """Hint of every window: the previous window's solution shifted by one period."""
    out = []
    for i, md in enumerate(models):
        if first[i] or results[i - 1].status != SolveStatus.kOptimal:
            out.append(None)
            continue
        PT = md.numVars() // 3
        T = md.numRows() - PT
        xs, ys = rolling_horizon_shift(results[i - 1].x, results[i - 1].y, T, PT // T)
        out.append(WarmStart(xs, ys, 0.0))
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--streams", type=int, default=2000)
    ap.add_argument("--windows", type=int, default=5)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--T", type=int, nargs=2, default=(24, 96))
    ap.add_argument("--P", type=int, nargs=2, default=(5, 20))
    ap.add_argument("--seed0", type=int, default=10000)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--label-batch", type=int, default=1024)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--tol", type=float, default=1e-6, help="relative KKT of the PDHG labels")
    ap.add_argument("--max-iterations", type=int, default=300000)
    ap.add_argument("--out", type=Path, default=DEFAULT_OUT)
    a = ap.parse_args(argv)
    o = PdhgOptions(tolerance=a.tol, max_iterations=a.max_iterations, check_frequency=64, algorithm=ALGO_HALPERN,
                    device=a.device)
    t0 = time.time()
    models, first = stream_windows(range(a.seed0, a.seed0 + a.streams), a.windows, tuple(a.T), tuple(a.P))
    results = []
    for k in range(0, len(models), a.label_batch):
        results += solve_batch(models[k:k + a.label_batch], o)
    t_label = time.time() - t0
    hints = shifted_hints(models, first, results)
    idx = [i for i in range(len(models)) if hints[i] is not None and results[i].status == SolveStatus.kOptimal]
    net = WarmStartNet(device=a.device, seed=0)
    rng = np.random.default_rng(0)
    idx = list(rng.permutation(idx))
    graphs = [net.graph([models[i] for i in idx[k:k + a.batch]],
                        training_targets([results[i] for i in idx[k:k + a.batch]]),
                        hints=[hints[i] for i in idx[k:k + a.batch]])
              for k in range(0, len(idx), a.batch)]
    t1 = time.time()
    hist = net.fit(graphs, epochs=a.epochs, lr=a.lr, lr_decay=0.97)
    t_train = time.time() - t1
    record = {"instances_solved": len(models), "instances_trained": len(idx), "streams": a.streams,
              "windows": a.windows, "T": list(a.T), "P": list(a.P), "epochs": a.epochs, "lr": a.lr,
              "label_s": t_label, "train_s": t_train, "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1],
              "optimal_labels": sum(r.status == SolveStatus.kOptimal for r in results), "label_tol": a.tol}
    a.out.parent.mkdir(parents=True, exist_ok=True)
    np.savez(a.out, params=net.params, record=json.dumps(record))
    print(json.dumps(record))


if __name__ == "__main__":
    main()
