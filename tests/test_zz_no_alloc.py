"""pramaan_spmv_noalloc: the allocation-free product for callers that cannot
call cudaMalloc where they need y = A x (fixed device-memory budgets, code
running under stream capture, hosts that own the memory pool).

The entry point is called through the C ABI on device buffers that the test
allocates beforehand.  Its output is compared with the oracle's restatement of
the reference's row loop (oracle.spmv_f32, src/gpu/pdhg_kernels.cuh:24-37) and
with the existing entry point (pramaan_launch_spmv), within the SpMV tolerance
the other tests use, |a - b| <= 1e-4 + 1e-4 * max(|a|, |b|), on two calls in a
row.  The shapes cover the kernel's paths: crossing rows, trailing empty rows,
a single tile, nnz an exact multiple of the 2048-entry tile, more tiles than
the grid (grid-stride loop), and tiles spanning more rows than the shared
row_ptr slice holds.  Collected last so a failure here leaves every other test
already run."""
import ctypes as C

import numpy as np
import pytest

import oracle
from lp_cases import random_csr
from pramaan_b200 import _lib as L
from pramaan_b200 import launch_spmv

pytestmark = pytest.mark.gpu

TILE = 2048


def close(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert a.shape == b.shape
    tol = 1e-4 + 1e-4 * np.maximum(np.abs(a), np.abs(b))
    bad = np.nonzero(~(np.abs(a - b) <= tol))[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}: {a[bad[:5]]} vs {b[bad[:5]]}"


def power_law_csr(seed, m=6000, n=20000):
    rng = np.random.default_rng(seed)
    k = np.arange(1, 6001)
    lengths = rng.choice(k, size=m, p=(k ** -1.5) / (k ** -1.5).sum())
    lengths[rng.random(m) < 0.05] = 0        # some empty rows
    lengths[7] = 5 * TILE + 3                 # a row over several 2048-entry tiles
    return random_csr(m, n, rng, lengths=lengths)


def csr_from_lengths(lengths, n, seed):
    """CSR with the given row lengths, uniform random columns (repeats allowed)."""
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, np.int64)
    rp = np.zeros(lengths.size + 1, np.int32)
    rp[1:] = np.cumsum(lengths)
    nnz = int(rp[-1])
    ci = rng.integers(0, n, size=nnz, dtype=np.int32)
    v = rng.standard_normal(nnz).astype(np.float32)
    return rp, ci, v


def call_noalloc(torch, rp, ci, v, x, m, n):
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(np.ascontiguousarray(rp, np.int32)).to(dev)
    d_ci = torch.from_numpy(np.ascontiguousarray(ci, np.int32)).to(dev)
    d_v = torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(dev)
    d_x = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dev)
    d_y = torch.full((m,), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    rc = L.lib().pramaan_spmv_noalloc(d_rp.data_ptr(), d_ci.data_ptr() if len(ci) else None,
                                      d_v.data_ptr() if len(v) else None, m, n, len(v),
                                      d_x.data_ptr(), d_y.data_ptr(), C.c_void_p(stream.cuda_stream))
    L.check(rc)
    torch.cuda.synchronize(dev)
    return d_y.cpu().numpy()


def check_twice(torch, rp, ci, v, m, n, seed, *, existing=True):
    """Two calls in a row with different x, each against the oracle (and the existing entry point)."""
    rng = np.random.default_rng(seed)
    rp, ci, v = (np.ascontiguousarray(a, t) for a, t in ((rp, np.int32), (ci, np.int32), (v, np.float32)))
    for _ in range(2):
        x = rng.standard_normal(n).astype(np.float32)
        y = call_noalloc(torch, rp, ci, v, x, m, n)
        close(y, oracle.spmv_f32(rp, ci, v, x, m))
        if existing:
            close(y, launch_spmv(rp, ci, v, x, m, n))


def test_noalloc_matches_oracle_and_existing_entry_point_twice():
    torch = pytest.importorskip("torch")
    rp, ci, v = power_law_csr(1)
    check_twice(torch, rp, ci, v, len(rp) - 1, 20000, seed=0)
    # a second matrix right after: the shared scratch holds the previous call's partials
    rp2, ci2, v2 = power_law_csr(2, m=3000, n=20000)
    check_twice(torch, rp2, ci2, v2, 3000, 20000, seed=1)


def test_noalloc_all_rows_empty():
    torch = pytest.importorskip("torch")
    m, n = 777, 50
    rp = np.zeros(m + 1, np.int32)
    for _ in range(2):
        y = call_noalloc(torch, rp, np.zeros(0, np.int32), np.zeros(0, np.float32),
                         np.ones(n, np.float32), m, n)
        assert np.array_equal(y, np.zeros(m, np.float32))


def test_noalloc_single_tile():
    torch = pytest.importorskip("torch")
    lengths = np.array([0, 3, 0, 700, 1, 0, 900, 2, 0, 0], np.int64)   # 1,606 entries
    rp, ci, v = csr_from_lengths(lengths, 300, seed=3)
    check_twice(torch, rp, ci, v, lengths.size, 300, seed=3)


def test_noalloc_exact_multiple_of_tile():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(4)
    lengths = rng.integers(0, 40, size=4000)
    lengths[-1] += 6 * TILE - int(lengths.sum()) % (6 * TILE)   # total a multiple of 6 tiles
    assert int(lengths.sum()) % TILE == 0
    rp, ci, v = csr_from_lengths(lengths, 5000, seed=4)
    check_twice(torch, rp, ci, v, lengths.size, 5000, seed=4)
    # and rows that end exactly on tile boundaries after crossing them
    lengths = np.array([TILE + 100, TILE - 100, 0, 0, 5 * TILE, 0], np.int64)
    rp, ci, v = csr_from_lengths(lengths, 1000, seed=5)
    check_twice(torch, rp, ci, v, lengths.size, 1000, seed=5)


def test_noalloc_trailing_empty_rows_after_crossing_row():
    torch = pytest.importorskip("torch")
    lengths = np.concatenate([np.full(50, 7), [3 * TILE + 11], np.zeros(300, np.int64)])
    rp, ci, v = csr_from_lengths(lengths, 4000, seed=6)
    check_twice(torch, rp, ci, v, lengths.size, 4000, seed=6)


def test_noalloc_more_tiles_than_grid():
    """nnz above 8 blocks per SM x 2048 entries: blocks take several tiles each."""
    torch = pytest.importorskip("torch")
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    rng = np.random.default_rng(7)
    m = 330_000
    lengths = rng.integers(0, 17, size=m)
    lengths[rng.integers(0, m, size=20)] = 9000   # long rows crossing tiles
    assert int(lengths.sum()) > 8 * sms * TILE
    rp, ci, v = csr_from_lengths(lengths, 1_000_000, seed=7)
    check_twice(torch, rp, ci, v, m, 1_000_000, seed=7)


def test_noalloc_tile_spanning_many_rows():
    """Tiles whose rows exceed the shared row_ptr slice (2,056 entries): row_ptr is read from global memory."""
    torch = pytest.importorskip("torch")
    m = 40_000
    lengths = np.zeros(m, np.int64)
    lengths[::2] = 1                     # alternating empty and one-entry rows: ~4,096 rows per tile
    lengths[25_001] = 3 * TILE           # and a crossing row among them
    rp, ci, v = csr_from_lengths(lengths, 2000, seed=8)
    check_twice(torch, rp, ci, v, m, 2000, seed=8)


def test_noalloc_allocates_no_device_memory():
    torch = pytest.importorskip("torch")
    rp, ci, v = power_law_csr(3)
    m, n = len(rp) - 1, 20000
    x = np.ones(n, np.float32)
    call_noalloc(torch, rp, ci, v, x, m, n)            # first call on the device: set-up
    dev = torch.device("cuda:0")
    bufs = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (rp, ci, v, x)]
    d_y = torch.empty(m, dtype=torch.float32, device=dev)
    torch.cuda.synchronize(dev)
    free0, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        L.check(L.lib().pramaan_spmv_noalloc(bufs[0].data_ptr(), bufs[1].data_ptr(), bufs[2].data_ptr(),
                                             m, n, len(v), bufs[3].data_ptr(), d_y.data_ptr(), None))
    torch.cuda.synchronize(dev)
    free1, _ = torch.cuda.mem_get_info(dev)
    assert free1 == free0


def test_noalloc_rejects_inputs_beyond_scratch_limit():
    limit = 65536 * 2048
    rc = L.lib().pramaan_spmv_noalloc(None, None, None, 10, 10, limit + 1, None, None, None)
    assert rc == L.PRAMAAN_ERR_INVALID_ARGUMENT
    assert b"exceeds the scratch limit" in L.lib().pramaan_last_error()
