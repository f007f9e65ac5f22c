"""pramaan_spmv_noalloc: the allocation-free product for callers that cannot
call cudaMalloc where they need y = A x (fixed device-memory budgets, code
running under stream capture, hosts that own the memory pool).

The entry point is called through the C ABI on device buffers that the test
allocates beforehand; its output is compared with the existing entry point
(pramaan_launch_spmv) within the SpMV tolerance the other tests use,
|a - b| <= 1e-4 + 1e-4 * max(|a|, |b|), on two calls in a row.  Collected last
so a failure here leaves every other test already run."""
import ctypes as C

import numpy as np
import pytest

from lp_cases import random_csr
from pramaan_b200 import _lib as L
from pramaan_b200 import launch_spmv

pytestmark = pytest.mark.gpu


def close(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    tol = 1e-4 + 1e-4 * np.maximum(np.abs(a), np.abs(b))
    bad = np.nonzero(np.abs(a - b) > tol)[0]
    assert bad.size == 0, f"{bad.size} mismatches, first {bad[:5]}: {a[bad[:5]]} vs {b[bad[:5]]}"


def power_law_csr(seed, m=6000, n=20000):
    rng = np.random.default_rng(seed)
    k = np.arange(1, 6001)
    lengths = rng.choice(k, size=m, p=(k ** -1.5) / (k ** -1.5).sum())
    lengths[rng.random(m) < 0.05] = 0        # some empty rows
    lengths[7] = 5 * 2048 + 3                 # a row over several 2048-entry tiles
    return random_csr(m, n, rng, lengths=lengths)


def call_noalloc(torch, rp, ci, v, x, m, n):
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(np.ascontiguousarray(rp, np.int32)).to(dev)
    d_ci = torch.from_numpy(np.ascontiguousarray(ci, np.int32)).to(dev)
    d_v = torch.from_numpy(np.ascontiguousarray(v, np.float32)).to(dev)
    d_x = torch.from_numpy(np.ascontiguousarray(x, np.float32)).to(dev)
    d_y = torch.full((m,), float("nan"), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    rc = L.lib().pramaan_spmv_noalloc(d_rp.data_ptr(), d_ci.data_ptr(), d_v.data_ptr(), m, n, len(v),
                                      d_x.data_ptr(), d_y.data_ptr(), C.c_void_p(stream.cuda_stream))
    L.check(rc)
    torch.cuda.synchronize(dev)
    return d_y.cpu().numpy()


def test_noalloc_matches_existing_entry_point_twice():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    rp, ci, v = power_law_csr(1)
    m, n = len(rp) - 1, 20000
    for call in range(2):   # two calls in a row, different x each time
        x = rng.standard_normal(n).astype(np.float32)
        close(call_noalloc(torch, rp, ci, v, x, m, n), launch_spmv(rp, ci, v, x, m, n))
    # a second matrix right after: the shared scratch holds the previous call's partials
    rp2, ci2, v2 = power_law_csr(2, m=3000, n=20000)
    x = rng.standard_normal(20000).astype(np.float32)
    close(call_noalloc(torch, rp2, ci2, v2, x, 3000, 20000), launch_spmv(rp2, ci2, v2, x, 3000, 20000))


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
