"""GPU tests of the restarted Halpern PDHG mode (PRAMAAN_ALGO_HALPERN).

The checker is the oracle's FP64 restatement oracle/adaptive.py
(solve_halpern).  The device runs FP32 corrections around FP64 master
iterates, so trajectories are not bit-identical; what is compared: the FP64
relative KKT of the answer (oracle.rel_kkt) meets the tolerance, the
objective equals the restatement's within the tolerance's reach, the
iteration counts agree within a factor of 2, and the mode needs fewer
iterations than the adaptive (PDLP-style) mode on the same LPs.
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN
from oracle import adaptive as oad
from pramaan_b200 import PdhgOptions, PdhgSolver, SolveStatus, solve_batch
from pramaan_b200.generators import ill_conditioned_lp, random_sparse_lp, rolling_horizon_batch, rolling_horizon_lp
from pramaan_b200.pdhg import ALGO_ADAPTIVE, ALGO_HALPERN

pytestmark = pytest.mark.gpu


def opts(tol, algo=ALGO_HALPERN, it=400000, refine=True):
    return PdhgOptions(tolerance=tol, max_iterations=it, check_frequency=64, algorithm=algo, refine=refine)


def lps():
    return {"rh24x5": rolling_horizon_lp(24, 5, seed=1), "rand300": random_sparse_lp(300, 900, 4, seed=0),
            "ill300": ill_conditioned_lp(300, 800, 4, seed=0, scale_exp=2), "wyndor": KNOWN["wyndor"][0]}


@pytest.mark.parametrize("tol", [1e-6, 1e-8])
def test_single_solves_match_the_restatement(tol):
    for name, md in lps().items():
        r = PdhgSolver(opts(tol)).solve(md)
        assert r.status == SolveStatus.kOptimal, (name, r.iterations)
        k = oracle.rel_kkt(md, r.x, r.y)
        assert max(k["primal"], k["dual"], k["gap"]) <= tol * 1.0001, (name, k)
        ref = oad.solve_halpern(md, tol=tol, max_iterations=400000)
        assert ref["status"] == "optimal"
        scale = 1 + abs(ref["kkt"]["pobj"])
        assert abs(k["pobj"] - ref["kkt"]["pobj"]) <= 20 * tol * scale, name
        assert 0.5 * ref["iterations"] <= r.iterations <= 2.0 * ref["iterations"] + 128, (name, r.iterations,
                                                                                          ref["iterations"])


def test_halpern_requires_fp64_master_iterates():
    with pytest.raises(ValueError, match="refine"):
        PdhgSolver(opts(1e-6, refine=False)).solve(random_sparse_lp(30, 90, 3, seed=1))


def test_batch_matches_single_solves_and_beats_the_adaptive_mode():
    models = rolling_horizon_batch(12, seed=3, T_range=(24, 60), P_range=(5, 12))
    hal = solve_batch(models, opts(1e-6))
    ada = solve_batch(models, opts(1e-6, ALGO_ADAPTIVE))
    for md, r in zip(models, hal):
        assert r.status == SolveStatus.kOptimal
        k = oracle.rel_kkt(md, r.x, r.y)
        assert max(k["primal"], k["dual"], k["gap"]) <= 1e-6 * 1.0001
        alone = PdhgSolver(opts(1e-6)).solve(md)
        assert r.objective_value == pytest.approx(alone.objective_value, rel=1e-4, abs=1e-4)
    assert sum(r.iterations for r in hal) < 0.8 * sum(r.iterations for r in ada)


def test_batch_is_deterministic_and_handles_early_answers():
    from pramaan_b200.pdhg import ModelIR
    models = rolling_horizon_batch(6, seed=4, T_range=(24, 40), P_range=(5, 8))
    empty = ModelIR([], [0, 0], [], [], [1.0], [2.0], [], [], 0, 4.5)
    a = solve_batch(models + [empty, KNOWN["wyndor"][0]], opts(1e-7))
    b = solve_batch(models + [empty, KNOWN["wyndor"][0]], opts(1e-7))
    for ra, rb in zip(a, b):
        assert ra.iterations == rb.iterations and np.array_equal(ra.x, rb.x)
    assert a[-2].status == SolveStatus.kOptimal and a[-2].objective_value == 4.5
    assert a[-1].objective_value == pytest.approx(36.0, rel=1e-6)


def test_warm_start_from_the_solution_stops_early():
    from pramaan_b200.gnn import training_targets
    models = rolling_horizon_batch(4, seed=5, T_range=(24, 30), P_range=(5, 6))
    cold = solve_batch(models, opts(1e-6))
    warm = solve_batch(models, opts(1e-6), warm=training_targets(cold))
    for c, w in zip(cold, warm):
        assert w.status == SolveStatus.kOptimal and w.iterations <= 64 < c.iterations


def test_interval_kernel_matches_the_per_kernel_path_bit_for_bit():
    """One cooperative kernel per check interval (persistent = 1) computes the
    same iterates as two launches per iteration in a CUDA graph
    (persistent = -1): every warp processes the same tiles with the same
    arithmetic.  The LPs include rows that cross tiles and an empty row, so
    the in-kernel fixups run."""
    from pramaan_b200.pdhg import ModelIR
    with_empty_row = ModelIR([1.0, 2.0, 1.0], [0, 2, 2, 4], [0, 1, 1, 2], [1.0, 1.0, 1.0, -1.0],
                             [1.0, -1e30, -2.0], [4.0, 5.0, 2.0], [0.0, 0.0, 0.0], [3.0, 3.0, 3.0], 0, 0.0)
    models = rolling_horizon_batch(5, seed=6, T_range=(24, 60), P_range=(5, 10)) + [
        random_sparse_lp(300, 900, 4, seed=2), with_empty_row]
    a = solve_batch(models, PdhgOptions(tolerance=1e-7, max_iterations=200000, check_frequency=64,
                                        algorithm=ALGO_HALPERN, persistent=1))
    b = solve_batch(models, PdhgOptions(tolerance=1e-7, max_iterations=200000, check_frequency=64,
                                        algorithm=ALGO_HALPERN, persistent=-1))
    for md, ra, rb in zip(models, a, b):
        assert ra.status == SolveStatus.kOptimal
        assert ra.iterations == rb.iterations and ra.restarts == rb.restarts
        assert np.array_equal(ra.x, rb.x) and np.array_equal(ra.y, rb.y)
    single = PdhgSolver(PdhgOptions(tolerance=1e-7, max_iterations=200000, check_frequency=37,
                                    algorithm=ALGO_HALPERN, persistent=1)).solve(models[5])
    single_g = PdhgSolver(PdhgOptions(tolerance=1e-7, max_iterations=200000, check_frequency=37,
                                      algorithm=ALGO_HALPERN, persistent=-1)).solve(models[5])
    assert single.iterations == single_g.iterations and np.array_equal(single.x, single_g.x)


def _with_empty_row():
    from pramaan_b200.pdhg import ModelIR
    return ModelIR([1.0, 2.0, 1.0], [0, 2, 2, 4], [0, 1, 1, 2], [1.0, 1.0, 1.0, -1.0],
                   [1.0, -1e30, -2.0], [4.0, 5.0, 2.0], [0.0, 0.0, 0.0], [3.0, 3.0, 3.0], 0, 0.0)


def test_cluster_kernel_follows_the_tiled_path():
    """One thread-block cluster per LP running whole check intervals
    (persistent = 2) against the tiled products in a CUDA graph
    (persistent = -1).  Both apply the same per-element updates; the cluster
    kernel sums each row in CSR order, which the tiled kernel also does for a
    row inside one tile, so over one check interval (no restart yet) the
    iterates agree to FP32 rounding, and complete solves reach the same
    certified answers."""
    models = rolling_horizon_batch(5, seed=6, T_range=(24, 60), P_range=(5, 10)) + [
        random_sparse_lp(300, 900, 4, seed=2), _with_empty_row()]
    short = dict(tolerance=0.0, max_iterations=64, check_frequency=64, algorithm=ALGO_HALPERN)
    a = solve_batch(models, PdhgOptions(persistent=2, **short))
    b = solve_batch(models, PdhgOptions(persistent=-1, **short))
    for ra, rb in zip(a, b):
        assert ra.iterations == rb.iterations == 64
        assert np.allclose(ra.x, rb.x, rtol=1e-4, atol=1e-4 * (1 + np.abs(rb.x).max()))
        assert np.allclose(ra.y, rb.y, rtol=1e-4, atol=1e-4 * (1 + np.abs(rb.y).max()))
    full = dict(tolerance=1e-7, max_iterations=200000, check_frequency=64, algorithm=ALGO_HALPERN)
    a = solve_batch(models, PdhgOptions(persistent=2, **full))
    b = solve_batch(models, PdhgOptions(persistent=-1, **full))
    for md, ra, rb in zip(models, a, b):
        assert ra.status == rb.status == SolveStatus.kOptimal
        k = oracle.rel_kkt(md, ra.x, ra.y)
        assert max(k["primal"], k["dual"], k["gap"]) <= 1e-7 * 1.0001
        assert ra.objective_value == pytest.approx(rb.objective_value, rel=1e-5, abs=1e-5)
        assert ra.iterations <= 2 * rb.iterations + 256 and rb.iterations <= 2 * ra.iterations + 256
    again = solve_batch(models, PdhgOptions(persistent=2, **full))
    for ra, rc in zip(a, again):   # deterministic run to run
        assert ra.iterations == rc.iterations and np.array_equal(ra.x, rc.x) and np.array_equal(ra.y, rc.y)


def _long_rows_and_columns_lp(seed=0):
    """400 x 1200 LP with three entries per column plus one row of 300
    entries, five rows of 40 and ten columns of 100 (rows and columns longer
    than the cluster kernel's one-thread limit of 16 entries, one past two
    64-entry warp steps), feasible and bounded by construction."""
    from pramaan_b200.generators import _csr_from_coo, _distinct_rows_per_col, _feasible_model

    rng = np.random.default_rng(seed)
    m, n = 400, 1200
    pairs = {(int(r), j) for j in range(n) for r in _distinct_rows_per_col(rng, m, 1, 3)[0]}
    pairs |= {(0, int(j)) for j in rng.choice(n, 300, replace=False)}
    for r in range(1, 6):
        pairs |= {(r, int(j)) for j in rng.choice(n, 40, replace=False)}
    for j in range(10):
        pairs |= {(int(r), j) for r in rng.choice(m, 100, replace=False)}
    rows = np.array([p[0] for p in pairs])
    cols = np.array([p[1] for p in pairs])
    vals = rng.standard_normal(rows.size)
    rp, ci, va = _csr_from_coo(rows, cols, vals, m)
    return _feasible_model(rng, m, n, rp, ci, va)[0]


def test_cluster_kernel_long_rows_and_columns():
    """Rows and columns past 16 entries go one warp each (lists built on the
    host); every row and column is still updated once per iteration, so the
    iterates follow the tiled path to FP32 rounding and the solve certifies."""
    md = _long_rows_and_columns_lp()
    lens = np.diff(np.asarray(md.row_ptr))
    assert lens.max() >= 300 and (np.bincount(np.asarray(md.col_idx)) > 16).sum() >= 10
    models = [md, random_sparse_lp(300, 900, 4, seed=2)]
    short = dict(tolerance=0.0, max_iterations=64, check_frequency=64, algorithm=ALGO_HALPERN)
    a = solve_batch(models, PdhgOptions(persistent=2, **short))
    b = solve_batch(models, PdhgOptions(persistent=-1, **short))
    for ra, rb in zip(a, b):
        assert np.allclose(ra.x, rb.x, rtol=1e-4, atol=1e-4 * (1 + np.abs(rb.x).max()))
        assert np.allclose(ra.y, rb.y, rtol=1e-4, atol=1e-4 * (1 + np.abs(rb.y).max()))
    full = dict(tolerance=1e-7, max_iterations=400000, check_frequency=64, algorithm=ALGO_HALPERN)
    r = solve_batch([md], PdhgOptions(persistent=2, **full))[0]
    assert r.status == SolveStatus.kOptimal
    k = oracle.rel_kkt(md, r.x, r.y)
    assert max(k["primal"], k["dual"], k["gap"]) <= 1e-7 * 1.0001


def test_cluster_kernel_single_lp_and_one_lp_left():
    """A single LP (a batch of one gets the largest cluster) and a batch whose
    compaction leaves one slow LP alone: answers certified and equal to the
    tiled path's within the tolerance's reach."""
    md = random_sparse_lp(1000, 3000, 4, seed=0)
    full = dict(tolerance=1e-8, max_iterations=400000, check_frequency=64, algorithm=ALGO_HALPERN)
    r = PdhgSolver(PdhgOptions(persistent=2, **full)).solve(md)
    g = PdhgSolver(PdhgOptions(persistent=-1, **full)).solve(md)
    assert r.status == g.status == SolveStatus.kOptimal
    k = oracle.rel_kkt(md, r.x, r.y)
    assert max(k["primal"], k["dual"], k["gap"]) <= 1e-8 * 1.0001
    assert r.objective_value == pytest.approx(g.objective_value, rel=1e-7, abs=1e-7)
    models = [rolling_horizon_lp(24, 5, seed=s) for s in range(6)] + [rolling_horizon_lp(96, 20, seed=7)]
    res = solve_batch(models, PdhgOptions(persistent=2, **dict(full, tolerance=1e-6)))
    for m_, rr in zip(models, res):
        assert rr.status == SolveStatus.kOptimal
        kk = oracle.rel_kkt(m_, rr.x, rr.y)
        assert max(kk["primal"], kk["dual"], kk["gap"]) <= 1e-6 * 1.0001
