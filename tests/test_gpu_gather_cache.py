"""Shared-memory gather cache (hot gather slots of an operand).

On an LP with power-law row lengths the transpose's gathers concentrate on
the long rows' y entries; the products keep those entries in shared memory.
Operands with local columns may instead have their gathers cached in L1.
The reference-mode cases run with the column-panel split off (panel_split
-1): they test the tiled kernels' gather modes, which the split would take
the longest rows away from (the split has its own tests, test_gpu_panel.py).
The value gathered is the same in every mode, so every iterate must be
bit-identical with the option gather_cache at 0 (automatic), 1 (L1-cached
gathers wherever there are no hot slots) and -1 (plain L2 gathers), in the
reference iteration (FP32 products, FP64 residual products with the FP32
remainders) and in the Halpern mode (FP64 master gathers through the slot
table).
"""
from __future__ import annotations

import numpy as np
import pytest

from pramaan_b200 import PdhgOptions, PdhgSolver
from pramaan_b200 import generators as gen
from pramaan_b200.pdhg import ALGO_HALPERN, ALGO_REFERENCE, Session

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def zipf_mid():
    # ~10.8 M non-zeros: large enough for the cache, rows Zipf(1.5) up to 5,000 long
    return gen.zipf_lp(200_000, 500_000, seed=3, device="cuda")


def test_reference_iterates_identical_with_and_without_cache(zipf_mid):
    runs = {}
    for cache in (0, -1):
        o = PdhgOptions(tolerance=1e-12, max_iterations=1000, check_frequency=100, algorithm=ALGO_REFERENCE, panel_split=-1,
                        gather_cache=cache)
        with Session(zipf_mid, o) as s:
            slots = s.gather_slots()
            s.iterate(60)
            res = s.residuals()
            x, y = s.iterates()
        runs[cache] = (slots, res, x, y)
    slots_on, res_on, x_on, y_on = runs[0]
    slots_off, res_off, x_off, y_off = runs[-1]
    assert slots_off == (0, 0)
    assert slots_on[0] == 0             # columns are uniform: no hot targets in A
    assert 1000 < slots_on[1] <= 16384  # the long rows' y entries in A^T
    assert np.array_equal(x_on, x_off) and np.array_equal(y_on, y_off)
    assert res_on == res_off
    assert np.isfinite(x_on).all() and np.abs(y_on).max() > 0


def test_halpern_solve_identical_with_and_without_cache(zipf_mid):
    out = {}
    for cache in (0, -1):
        o = PdhgOptions(tolerance=1e-12, max_iterations=640, check_frequency=64, algorithm=ALGO_HALPERN,
                        gather_cache=cache)
        out[cache] = PdhgSolver(o).solve(zipf_mid)
    a, b = out[0], out[-1]
    assert a.iterations == b.iterations
    assert a.status == b.status
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
    assert a.objective_value == b.objective_value


def test_gather_cache_option_is_validated():
    md = gen.random_sparse_lp(50, 120, 4, seed=1)
    with pytest.raises(ValueError):
        PdhgSolver(PdhgOptions(gather_cache=2)).solve(md)


@pytest.fixture(scope="module")
def banded_mid():
    # ~10.7 M non-zeros, every row's columns within +-256 of i*n/m: local gathers, no hot targets
    return gen.banded_lp(400_000, 1_000_000, per_row=27, band=256, seed=2, device="cuda")


def test_l1_cached_gathers_identical_to_l2_gathers(banded_mid):
    runs = {}
    for cache in (1, 0, -1):
        o = PdhgOptions(tolerance=1e-12, max_iterations=1000, check_frequency=100, algorithm=ALGO_REFERENCE, panel_split=-1,
                        gather_cache=cache)
        with Session(banded_mid, o) as s:
            info = s.gather_info()
            s.iterate(40)
            res = s.residuals()
            x, y = s.iterates()
        runs[cache] = (info, res, x, y)
    forced, auto, off = runs[1], runs[0], runs[-1]
    for op in ("A", "AT"):
        assert (forced[0][op]["hot_slots"], forced[0][op]["l1"]) == (0, True)
        assert (off[0][op]["hot_slots"], off[0][op]["l1"]) == (0, False)
    assert auto[0]["A"]["hot_slots"] == 0 and auto[0]["AT"]["hot_slots"] == 0
    for run in (forced, auto):
        assert np.array_equal(run[2], off[2]) and np.array_equal(run[3], off[3])
        assert run[1] == off[1]


def test_halpern_with_hot_slots_and_l1_gathers_identical(zipf_mid):
    out = {}
    for cache in (1, -1):
        o = PdhgOptions(tolerance=1e-12, max_iterations=320, check_frequency=64, algorithm=ALGO_HALPERN,
                        gather_cache=cache)
        out[cache] = PdhgSolver(o).solve(zipf_mid)
    a, b = out[1], out[-1]
    assert a.iterations == b.iterations
    assert np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


def _with_empty_rows_and_columns(md):
    """The LP with the entries of every 7th column and every 11th row removed,
    so both operands compact empty rows away (row maps) while A^T keeps its
    hot targets."""
    from pramaan_b200.pdhg import ModelIR

    rows = np.repeat(np.arange(md.numRows()), np.diff(md.row_ptr))
    keep = (md.col_idx % 7 != 0) & (rows % 11 != 0)
    rp = np.zeros(md.numRows() + 1, np.int64)
    np.cumsum(np.bincount(rows[keep], minlength=md.numRows()), out=rp[1:])
    return ModelIR(md.obj_coeffs, rp, md.col_idx[keep], md.values[keep], md.row_lower, md.row_upper,
                   md.var_lower, md.var_upper, md.obj_sense, md.obj_offset)


def test_hot_slots_with_row_maps_identical(zipf_mid):
    md = _with_empty_rows_and_columns(zipf_mid)
    runs = {}
    for cache in (0, 1, -1):
        o = PdhgOptions(tolerance=1e-12, max_iterations=1000, check_frequency=100, algorithm=ALGO_REFERENCE, panel_split=-1,
                        gather_cache=cache)
        with Session(md, o) as s:
            info = s.gather_info()
            s.iterate(40)
            res = s.residuals()
            x, y = s.iterates()
        runs[cache] = (info, res, x, y)
    assert runs[0][0]["AT"]["hot_slots"] > 1000 and runs[-1][0]["AT"]["hot_slots"] == 0
    assert runs[1][0]["A"]["l1"]
    for cache in (0, 1):
        assert np.array_equal(runs[cache][2], runs[-1][2]) and np.array_equal(runs[cache][3], runs[-1][3])
        assert runs[cache][1] == runs[-1][1]
    # the emptied columns keep their clamped start; the emptied rows move only with their bounds
    assert np.isfinite(runs[0][2]).all()


@pytest.mark.parametrize("blocks", [1, 3, 5])
def test_launch_shape_changes_no_iterate(blocks):
    """The launch shape (`launch_blocks`: resident blocks per SM; above 3 the
    dense variants, which stage finished rows over the tile's own slots)
    only moves tiles between warps: every tile is summed by the same code and
    rows crossing tiles are completed in tile order.  On a banded LP large
    enough for the autotuner, the iterates after 40 reference iterations, the
    FP64 residuals and a Halpern solve are bit-identical to the autotuned
    launch's, with L1-cached and with L2 gathers."""
    md = gen.banded_lp(200_000, 500_000, per_row=24, band=128, seed=5)
    for cache in (1, -1):
        runs = []
        for lb in (0, blocks):
            o = PdhgOptions(tolerance=1e-12, max_iterations=1000, check_frequency=100, algorithm=ALGO_REFERENCE, panel_split=-1,
                            gather_cache=cache, launch_blocks=lb)
            with Session(md, o) as s:
                s.iterate(40)
                runs.append((s.residuals(), *s.iterates()))
        (r0, x0, y0), (r1, x1, y1) = runs
        assert np.array_equal(x0, x1) and np.array_equal(y0, y1) and r0 == r1
    h = [PdhgSolver(PdhgOptions(tolerance=1e-12, max_iterations=256, check_frequency=64, algorithm=ALGO_HALPERN,
                                launch_blocks=lb)).solve(md) for lb in (0, blocks)]
    assert h[0].iterations == h[1].iterations and np.array_equal(h[0].x, h[1].x)
