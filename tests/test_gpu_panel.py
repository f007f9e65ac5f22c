"""Column-panel split of the products (csrc/panel.cuh, panel.cu).

The long rows of A are computed over column panels of x̄ held in shared
memory (one per SM) and their per-panel partial sums added in panel order;
the short rows keep the tiled product.  The longest rows' part of Aᵀy runs
over the same panels (every block holds those rows' y, one segment per
column) and the tiled Aᵀy over the other entries adds it.  The splits change
only the order of the additions, so:
  * iterates after k reference iterations match the oracle's restatement of
    the reference iteration (src/gpu/pdhg_kernels.cuh:24-109) within
    |gpu - ref| <= 1e-4 * (1 + |ref|), the tolerance of the tiled product's
    trajectory test;
  * every sum has a fixed order: two runs give bit-identical iterates;
  * they match the tiled product alone (panel_split -1) within the same
    tolerance.
Edge cases: every row long (min length 2, most segments empty, chunks closed
by the segment cap), empty rows, rows longer than a chunk spread over
panels, fewer columns than SMs (narrow panels), and a row whose entries in
one panel exceed a chunk (the split is then declined and the tiled product
runs).
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle
from lp_cases import random_csr
from pramaan_b200 import PdhgOptions, PdhgSolver, Session
from pramaan_b200.generators import zipf_lp
from pramaan_b200.pdhg import ModelIR, ObjSense

pytestmark = pytest.mark.gpu


def _feasible(rp, ci, v, m, n, seed):
    """Feasible LP on a given CSR (the benchmark generators' construction:
    b = A x0, c = A^T y0 + s0, 0 <= x <= x0 + U(1, 5))."""
    rng = np.random.default_rng(seed)
    rows = np.repeat(np.arange(m), np.diff(rp))
    vals = v.astype(np.float64)
    x0 = rng.random(n)
    b = np.bincount(rows, weights=vals * x0[ci], minlength=m)
    y0 = rng.standard_normal(m)
    c = np.bincount(ci, weights=vals * y0[rows], minlength=n) + rng.random(n)
    u = x0 + rng.uniform(1.0, 5.0, size=n)
    return ModelIR(c, rp.astype(np.int32), ci.astype(np.int32), vals, b, b.copy(), np.zeros(n), u,
                   ObjSense.kMinimize, 0.0)


def _run(model, k, split):
    with Session(model, PdhgOptions(panel_split=split)) as s:
        info = s.panel_info()
        s.iterate(k)
        x, y = s.iterates()
    return info, x, y


def _check_oracle(model, k, x, y, name):
    rx, ry, _ = oracle.trajectory(model, k)
    np.testing.assert_allclose(x, rx, rtol=1e-4, atol=1e-4, err_msg=f"{name} x after {k}")
    np.testing.assert_allclose(y, ry, rtol=1e-4, atol=1e-4 * (1 + np.abs(ry).max()), err_msg=f"{name} y after {k}")


@pytest.fixture(scope="module")
def zipf_small():
    # 20,000 x 300,000, Zipf(1.5) rows up to 5,000 long: ~1 M non-zeros, ~89 % in rows of >= 74
    return zipf_lp(20_000, 300_000, cap=5000, seed=5)


@pytest.mark.parametrize("k", [1, 20])
def test_panel_trajectory_matches_oracle(zipf_small, k):
    info, x, y = _run(zipf_small, k, 1)
    assert info["panels"] > 100 and info["long_rows"] > 0
    assert info["long_nnz"] > 0.5 * zipf_small.nnz()
    # the longest rows' part of A^T y runs over the same panels
    assert info["primal_hot_rows"] > 0 and info["primal_hot_nnz"] > 0.5 * zipf_small.nnz()
    _check_oracle(zipf_small, k, x, y, "zipf 20k x 300k")


def test_panel_deterministic_and_matches_tiled(zipf_small):
    _, x1, y1 = _run(zipf_small, 30, 1)
    _, x2, y2 = _run(zipf_small, 30, 1)
    assert np.array_equal(x1, x2) and np.array_equal(y1, y2)
    info, xt, yt = _run(zipf_small, 30, -1)
    assert info["panels"] == 0 and info["primal_hot_rows"] == 0
    np.testing.assert_allclose(x1, xt, rtol=1e-4, atol=1e-4)
    np.testing.assert_allclose(y1, yt, rtol=1e-4, atol=1e-4 * (1 + np.abs(yt).max()))


def _mixed_lp(seed, m=3000, n=50_000):
    """Poisson(4) rows, 5 % emptied, 60 rows of 300-3,000 entries."""
    rng = np.random.default_rng(seed)
    long_rows = {int(r): int(L) for r, L in zip(rng.choice(m, 60, replace=False), rng.integers(300, 3000, 60))}
    rp, ci, v = random_csr(m, n, rng, empty_frac=0.05, long_rows=long_rows)
    return _feasible(rp, ci, v, m, n, seed)


@pytest.mark.parametrize("min_len", [2, 40, 400])
def test_panel_long_row_sets(min_len):
    model = _mixed_lp(11)
    info, x, y = _run(model, 12, min_len)
    assert info["panels"] > 0 and info["min_len"] == min_len
    assert info["primal_hot_rows"] == int((np.diff(model.row_ptr) >= 32).sum())   # rows of >= 32 entries
    lens = np.diff(model.row_ptr)
    assert info["long_rows"] == int((lens >= min_len).sum())
    _check_oracle(model, 12, x, y, f"mixed, long rows >= {min_len}")


def test_panel_narrow_panels():
    # 100 columns: panels of 4 columns, fewer panels than SMs
    m, n = 2000, 100
    rng = np.random.default_rng(3)
    rp, ci, v = random_csr(m, n, rng, lengths=rng.integers(0, 60, m))
    model = _feasible(rp, ci, v, m, n, 3)
    info, x, y = _run(model, 15, 2)
    assert 0 < info["panels"] <= 100
    # about 400 hot entries per column: more than a chunk, so A^T y stays tiled
    assert info["primal_hot_rows"] == 0
    _check_oracle(model, 15, x, y, "narrow panels")


def test_panel_declined_when_a_segment_exceeds_a_chunk():
    # one row with 600 entries in the first 600 columns: 600 > 512 entries in one panel
    m, n = 500, 148 * 1000
    rng = np.random.default_rng(4)
    rp, ci, v = random_csr(m, n, rng, lengths=rng.integers(1, 300, m))
    lens = np.diff(rp).copy()
    lens[0] = 600
    cols = [np.arange(600)] + [ci[rp[i]:rp[i + 1]] for i in range(1, m)]
    vals = [rng.standard_normal(600).astype(np.float32)] + [v[rp[i]:rp[i + 1]] for i in range(1, m)]
    rp2 = np.zeros(m + 1, np.int64)
    rp2[1:] = np.cumsum(lens)
    model = _feasible(rp2, np.concatenate(cols), np.concatenate(vals), m, n, 4)
    info, x, y = _run(model, 10, 1)
    assert info["panels"] == 0   # declined: the tiled product runs
    _check_oracle(model, 10, x, y, "declined split")


def test_panel_solve_matches_tiled_solve(zipf_small):
    out = {}
    for split in (1, -1):
        o = PdhgOptions(tolerance=1e-12, max_iterations=400, check_frequency=100, panel_split=split)
        out[split] = PdhgSolver(o).solve(zipf_small)
    a, b = out[1], out[-1]
    assert a.status == b.status and a.iterations == b.iterations
    assert a.objective_value == pytest.approx(b.objective_value, rel=1e-4, abs=1e-4)
    np.testing.assert_allclose(a.x, b.x, rtol=1e-4, atol=1e-4)
