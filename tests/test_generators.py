"""CPU checks of the seeded workload generators (shapes of the benchmark
configurations) — structure, feasibility by construction, determinism."""
import numpy as np
import pytest

import oracle
from pramaan_b200.generators import (random_sparse_lp, rolling_horizon_batch, rolling_horizon_lp,
                                    rolling_horizon_shift, rolling_horizon_tail_mask)


def test_rolling_horizon_structure():
    T, P = 7, 3
    m = rolling_horizon_lp(T, P, seed=5)
    PT = P * T
    assert (m.numRows(), m.numVars()) == (PT + T, 3 * PT)
    assert m.nnz() == 6 * PT - 2 * P
    # balance rows are equalities on the demand, capacity rows are <= cap
    np.testing.assert_array_equal(m.row_lower[:PT], m.row_upper[:PT])
    assert np.all(m.row_lower[PT:] <= -1e29) and np.all(m.row_upper[PT:] > 0)
    assert np.all(m.var_lower == 0) and np.all(m.var_upper >= 1e29)
    assert np.all((m.obj_coeffs >= 1) & (m.obj_coeffs <= 10))
    # columns sorted within rows, values +-1
    for i in range(m.numRows()):
        c = m.col_idx[m.row_ptr[i]:m.row_ptr[i + 1]]
        assert np.all(np.diff(c) > 0)
    assert set(np.unique(m.values)) <= {-1.0, 1.0}


def test_rolling_horizon_feasible_point_by_backlog():
    # produce nothing, backlog everything: B[p,t] = cumulative demand is feasible
    T, P = 6, 2
    m = rolling_horizon_lp(T, P, seed=1)
    d = m.row_lower[:P * T].reshape(P, T)
    x = np.zeros(m.numVars())
    x[2 * P * T:] = np.cumsum(d, axis=1).ravel()
    act = m.multiply(x)
    np.testing.assert_allclose(act[:P * T], d.ravel(), rtol=1e-12, atol=1e-9)
    assert np.all(act[P * T:] <= m.row_upper[P * T:])


def test_rolling_horizon_batch_shapes_and_determinism():
    a = rolling_horizon_batch(20, seed=3)
    b = rolling_horizon_batch(20, seed=3)
    for x, y in zip(a, b):
        assert x.numVars() == y.numVars() and np.array_equal(x.obj_coeffs, y.obj_coeffs)
    T = [(x.numRows() - x.numVars() // 3) for x in a]          # m - PT = T
    assert min(T) >= 24 and max(T) <= 336
    P = [x.numVars() // 3 // t for x, t in zip(a, T)]
    assert min(P) >= 5 and max(P) <= 50


@pytest.mark.skipif(oracle.ref_cpu() is None, reason="oracle/_ref not built (needs the reference tree)")
def test_rolling_horizon_small_solved_by_reference_simplex():
    m = rolling_horizon_lp(4, 2, seed=8)
    cpu = oracle.ref_solve("simplex", m, max_iterations=100000)
    assert cpu["status"] == 0
    assert oracle.certificate(m, cpu["x"])["primal_residual"] <= 1e-6


def test_random_sparse_lp_feasible_by_construction():
    m, cert = random_sparse_lp(50, 150, 4, seed=2, return_certificate=True)
    np.testing.assert_allclose(m.multiply(cert["x0"]), m.row_lower, rtol=1e-12, atol=1e-9)


def test_rolling_horizon_tail_mask_and_splice():
    """The tail mask selects the last k periods of every block of the
    rolling-horizon layout (three variable blocks of P x T, P balance rows of
    T, then T capacity rows); the spliced start takes the network's values
    there and the hint's elsewhere.  The period the shift only copies is
    always inside a non-empty tail."""
    from pramaan_b200.gnn import WarmStart, splice_refinement

    T, P = 7, 3
    md = rolling_horizon_lp(T, P, seed=1)
    assert md.numVars() == 3 * P * T and md.numRows() == P * T + T
    xm, ym = rolling_horizon_tail_mask(T, P, 2)
    assert xm.shape == (3 * P * T,) and ym.shape == (P * T + T,)
    t = np.tile(np.arange(T), 3 * P)
    assert np.array_equal(xm, t >= T - 2)
    assert np.array_equal(ym, np.concatenate([np.tile(np.arange(T), P), np.arange(T)]) >= T - 2)
    assert not rolling_horizon_tail_mask(T, P, 0)[0].any() and rolling_horizon_tail_mask(T, P, 99)[1].all()
    rng = np.random.default_rng(0)
    x, y = rng.standard_normal(3 * P * T), rng.standard_normal(P * T + T)
    xs, ys = rolling_horizon_shift(x, y, T, P)
    copied = np.tile(np.arange(T), 3 * P) == T - 1
    assert np.array_equal(xs[copied], x[np.tile(np.arange(T), 3 * P) == T - 1])
    assert xm[copied].all()
    hint = WarmStart(xs, ys, 0.0)
    pred = WarmStart(rng.standard_normal(xs.size), rng.standard_normal(ys.size), 2.0)
    sp = splice_refinement(hint, pred, (xm, ym))
    assert np.array_equal(sp.x, np.where(xm, pred.x, xs)) and np.array_equal(sp.y, np.where(ym, pred.y, ys))
    assert sp.primal_weight == 0.0
    assert splice_refinement(hint, pred, None) is pred and splice_refinement(None, pred, (xm, ym)) is pred
