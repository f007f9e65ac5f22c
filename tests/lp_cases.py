"""LP fixtures shared by the tests.

The small LPs with known optima restate the cases of the reference's GPU
test (tests/test_gpu_pdhg.cpp:263-404); the matrix builders mirror its
denseToCSR helper (:88-103).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from pramaan_b200.pdhg import ModelIR, ObjSense, kInfinity as INF

REPO = Path(__file__).resolve().parent.parent
MPS_DIR = REPO / "oracle" / "_ref" / "run" / "tests" / "data"


def dense_to_csr(rows, n):
    rp, ci, v = [0], [], []
    for r in rows:
        for j in range(n):
            if r[j] != 0.0:
                ci.append(j)
                v.append(float(r[j]))
        rp.append(len(ci))
    return rp, ci, v


def lp(sense, offset, c, A, n, rl, ru, vl, vu) -> ModelIR:
    rp, ci, v = dense_to_csr(A, n)
    return ModelIR(c, rp, ci, v, rl, ru, vl, vu, sense, offset)


MIN, MAX = ObjSense.kMinimize, ObjSense.kMaximize

# name -> (model, known objective or None, check feasibility)
KNOWN = {
    # max 3x1 + 5x2, x1<=4, 2x2<=12, 3x1+2x2<=18  -> 36 at (2, 6)
    "wyndor": (lp(MAX, 0.0, [3, 5], [[1, 0], [0, 2], [3, 2]], 2, [-INF] * 3, [4, 12, 18],
                  [0, 0], [INF, INF]), 36.0, True),
    # min 2x - y + 10, no rows, x in [0,10], y in [-5,5] -> 5
    "zero_row": (lp(MIN, 10.0, [2, -1], [], 2, [], [], [0, -5], [10, 5]), 5.0, False),
    # min x, x >= 3 -> 3
    "one_var": (lp(MIN, 0.0, [1], [[1]], 1, [3], [INF], [0], [INF]), 3.0, True),
    # min x+y, x+y = 5 -> 5
    "equality": (lp(MIN, 0.0, [1, 1], [[1, 1]], 2, [5], [5], [0, 0], [INF, INF]), 5.0, True),
    # min -x1-2x2, x1+x2<=4, x1<=3, x2<=3 -> -7
    "multi": (lp(MIN, 0.0, [-1, -2], [[1, 1], [1, 0], [0, 1]], 2, [-INF] * 3, [4, 3, 3],
                 [0, 0], [INF, INF]), -7.0, True),
    # min 0, x+y>=2 -> 0
    "zero_obj": (lp(MIN, 0.0, [0, 0], [[1, 1]], 2, [2], [INF], [0, 0], [INF, INF]), 0.0, True),
    # min x+y, x+y<=10, x in [2,5], y in [3,7] -> 5
    "bounded": (lp(MIN, 0.0, [1, 1], [[1, 1]], 2, [-INF], [10], [2, 3], [5, 7]), 5.0, True),
    # Wyndor again, built from a dense matrix with structural zeros
    "sparse_zeros": (lp(MAX, 0.0, [3, 5], [[1, 0], [0, 2], [3, 2]], 2, [-INF] * 3, [4, 12, 18],
                        [0, 0], [INF, INF]), 36.0, False),
}

# min 1e-3 x + 1e3 y, 1e3 x + 1e-3 y >= 1: only termination is required.
SCALED = lp(MIN, 0.0, [1e-3, 1e3], [[1e3, 1e-3]], 2, [1.0], [INF], [0, 0], [INF, INF])


def primal_violation(model: ModelIR, x) -> float:
    """Max bound and row violation (tests/test_gpu_pdhg.cpp:106-118)."""
    x = np.asarray(x, np.float64)
    v = 0.0
    if x.size:
        v = max(v, float(np.max(np.maximum(model.var_lower - x, 0.0))),
                float(np.max(np.maximum(x - model.var_upper, 0.0))))
    if model.numRows():
        act = model.multiply(x)
        v = max(v, float(np.max(np.maximum(model.row_lower - act, 0.0))),
                float(np.max(np.maximum(act - model.row_upper, 0.0))))
    return v


def random_csr(m: int, n: int, rng: np.random.Generator, *, lengths=None, empty_frac=0.0,
               long_rows=()):
    """Random FP32 CSR with distinct sorted columns per row.

    `lengths`: per-row lengths (default Poisson(4) clipped to n); rows picked
    with probability `empty_frac` are emptied; `long_rows` forces given rows
    to the given lengths ({row: length})."""
    if lengths is None:
        lengths = np.minimum(rng.poisson(4.0, size=m), n)
    lengths = np.asarray(lengths, np.int64).copy()
    if empty_frac > 0:
        lengths[rng.random(m) < empty_frac] = 0
    for r, L in dict(long_rows).items():
        lengths[r] = min(L, n)
    cols = []
    for L in lengths:
        cols.append(np.sort(rng.choice(n, size=int(L), replace=False)) if L else np.zeros(0, np.int64))
    rp = np.zeros(m + 1, np.int32)
    rp[1:] = np.cumsum(lengths)
    ci = np.concatenate(cols).astype(np.int32) if m else np.zeros(0, np.int32)
    v = rng.standard_normal(ci.size).astype(np.float32)
    return rp, ci, v


def mps_model(name: str) -> ModelIR | None:
    """afiro / adlittle through the reference's own MPS parser (oracle/_ref)."""
    import oracle

    path = MPS_DIR / f"{name}.mps"
    if not path.exists() or oracle.ref_cpu() is None:
        return None
    return oracle.ref_load_mps(str(path))
