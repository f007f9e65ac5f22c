"""GPU parity of the SpMV pair against the oracle, through the C ABI
(pramaan_launch_spmv / pramaan_launch_spmv_t).

Tolerance: |gpu - ref| <= 1e-4 + 1e-4 * max(|gpu|, |ref|) per element, the
reference's own SpMV test tolerance (tests/test_gpu_pdhg.cpp:191-193).  The
oracle sums each row sequentially; the kernel sums in tile/scan order, so the
comparison is within tolerance, not bitwise.  Run-to-run results of the
kernel must be bitwise identical (no atomics in the sums).
"""
import numpy as np
import pytest

import oracle
from lp_cases import random_csr
from pramaan_b200 import launch_spmv, launch_spmv_t

pytestmark = pytest.mark.gpu
TILE = 512


def close(gpu, ref):
    gpu, ref = np.asarray(gpu, np.float64), np.asarray(ref, np.float64)
    assert gpu.shape == ref.shape
    tol = 1e-4 + 1e-4 * np.maximum(np.abs(gpu), np.abs(ref))
    bad = np.nonzero(np.abs(gpu - ref) > tol)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first at {bad[:5]}: gpu={gpu[bad[:5]]} ref={ref[bad[:5]]}"


def both(rp, ci, v, m, n, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n).astype(np.float32)
    xt = rng.standard_normal(m).astype(np.float32)
    close(launch_spmv(rp, ci, v, x, m, n), oracle.spmv_f32(rp, ci, v, x, m))
    close(launch_spmv_t(rp, ci, v, xt, m, n), oracle.spmv_t_f32(rp, ci, v, xt, m, n))


@pytest.mark.parametrize("d", [1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129])
def test_reference_diagonal_dimensions(d):
    # tests/test_gpu_pdhg.cpp:236-245: A = diag(1..d), x_j = (j+1)/2
    rp = np.arange(d + 1, dtype=np.int32)
    ci = np.arange(d, dtype=np.int32)
    v = np.arange(1, d + 1, dtype=np.float32)
    x = (np.arange(d, dtype=np.float32) + 1) * np.float32(0.5)
    close(launch_spmv(rp, ci, v, x, d, d), oracle.spmv_f32(rp, ci, v, x, d))
    xt = (np.arange(d, dtype=np.float32) + 1) * np.float32(0.3)
    close(launch_spmv_t(rp, ci, v, xt, d, d), oracle.spmv_t_f32(rp, ci, v, xt, d, d))


def test_reference_rectangle_and_empty():
    rp = np.array([0, 2, 3, 5], np.int32)
    ci = np.array([1, 5, 3, 0, 6], np.int32)
    v = np.array([2, -1, 3, 1, 4], np.float32)
    both(rp, ci, v, 3, 7)
    # m = 0 (tests/test_gpu_pdhg.cpp:256-257)
    assert launch_spmv(np.zeros(1, np.int32), [], [], np.ones(5, np.float32), 0, 5).size == 0
    np.testing.assert_array_equal(launch_spmv_t(np.zeros(1, np.int32), [], [], [], 0, 5), np.zeros(5))


@pytest.mark.parametrize("m,n,seed", [(1, 1, 0), (7, 3, 1), (300, 200, 2), (5000, 4000, 3),
                                      (20000, 300, 4)])
def test_random_poisson_rows(m, n, seed):
    rp, ci, v = random_csr(m, n, np.random.default_rng(seed))
    both(rp, ci, v, m, n, seed)


def test_empty_rows_everywhere():
    rng = np.random.default_rng(11)
    m, n = 6000, 900
    rp, ci, v = random_csr(m, n, rng, empty_frac=0.4)
    # leading and trailing empty rows too
    lengths = np.diff(rp)
    lengths[:17] = 0
    lengths[-23:] = 0
    rp2 = np.zeros(m + 1, np.int32)
    rp2[1:] = np.cumsum(lengths)
    keep = np.concatenate([np.arange(rp[i], rp[i] + lengths[i]) for i in range(m)]).astype(np.int64)
    both(rp2, ci[keep], v[keep], m, n)


def test_rows_spanning_many_tiles():
    rng = np.random.default_rng(5)
    m, n = 40, 60000
    lengths = rng.integers(0, 50, size=m)
    lengths[3] = 5 * TILE + 17      # spans six tiles
    lengths[4] = TILE               # exactly one tile
    lengths[20] = 3 * TILE - 1
    lengths[39] = 2 * TILE + 1      # last row crosses into the pad
    rp, ci, v = random_csr(m, n, rng, lengths=lengths)
    both(rp, ci, v, m, n)


def test_nnz_exact_tile_multiple_and_single_row():
    rng = np.random.default_rng(9)
    rp, ci, v = random_csr(1, 3 * TILE, rng, lengths=[3 * TILE])
    both(rp, ci, v, 1, 3 * TILE)
    lengths = np.full(TILE // 4, 4)
    rp, ci, v = random_csr(TILE // 4, 50, rng, lengths=lengths)   # nnz == TILE exactly
    assert rp[-1] == TILE
    both(rp, ci, v, TILE // 4, 50)


def test_power_law_rows():
    rng = np.random.default_rng(21)
    m, n = 20000, 50000
    k = np.arange(1, 5001)
    p = k ** -1.5
    lengths = rng.choice(k, size=m, p=p / p.sum())
    rp, ci, v = random_csr(m, n, rng, lengths=lengths)
    both(rp, ci, v, m, n)


def test_deterministic_bitwise():
    rng = np.random.default_rng(2)
    m, n = 30000, 20000
    k = np.arange(1, 3000)
    lengths = rng.choice(k, size=m, p=(k ** -1.5) / (k ** -1.5).sum())
    rp, ci, v = random_csr(m, n, rng, lengths=lengths)
    x = rng.standard_normal(n).astype(np.float32)
    xt = rng.standard_normal(m).astype(np.float32)
    a1, a2 = launch_spmv(rp, ci, v, x, m, n), launch_spmv(rp, ci, v, x, m, n)
    t1, t2 = launch_spmv_t(rp, ci, v, xt, m, n), launch_spmv_t(rp, ci, v, xt, m, n)
    assert np.array_equal(a1.view(np.uint32), a2.view(np.uint32))
    assert np.array_equal(t1.view(np.uint32), t2.view(np.uint32))


def test_invalid_structure_rejected():
    with pytest.raises(ValueError, match="col_idx"):
        launch_spmv(np.array([0, 1], np.int32), np.array([5], np.int32), np.ones(1, np.float32),
                    np.ones(3, np.float32), 1, 3)
    with pytest.raises(ValueError, match="row_ptr"):
        launch_spmv(np.array([0, 2, 1], np.int32), np.array([0], np.int32), np.ones(1, np.float32),
                    np.ones(3, np.float32), 2, 3)
