"""Device memory cache: solves allocate their operands and temporaries from a
per-device cache that keeps freed blocks for reuse (cudaFree's device
synchronisation kept).  Repeated solves must give identical answers whether
their buffers are new or reused, and releasing the cache must leave the
library working."""
from __future__ import annotations

import numpy as np
import pytest

from pramaan_b200 import PdhgOptions, PdhgSolver, release_cached_memory, solve_batch
from pramaan_b200 import generators as gen
from pramaan_b200.pdhg import ALGO_HALPERN

pytestmark = pytest.mark.gpu


def test_reused_buffers_give_identical_solves():
    md = gen.random_sparse_lp(400, 1200, 4, seed=7)
    o = PdhgOptions(tolerance=1e-6, max_iterations=20000)
    release_cached_memory()
    first = PdhgSolver(o).solve(md)            # fresh allocations
    again = PdhgSolver(o).solve(md)            # the same sizes, from the cache
    release_cached_memory(0)
    after = PdhgSolver(o).solve(md)            # fresh again
    for r in (again, after):
        assert r.status == first.status and r.iterations == first.iterations
        assert np.array_equal(r.x, first.x) and np.array_equal(r.y, first.y)


def test_cache_across_batches_of_different_sizes():
    o = PdhgOptions(tolerance=1e-6, max_iterations=100000, check_frequency=64, algorithm=ALGO_HALPERN)
    big = [gen.rolling_horizon_lp(48, 8, seed=s) for s in range(6)]
    small = big[:2]
    ref = solve_batch(small, o)
    solve_batch(big, o)                        # larger blocks enter the cache
    again = solve_batch(small, o)              # served from larger cached blocks
    for a, b in zip(ref, again):
        assert a.iterations == b.iterations and np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)


def test_release_rejects_bad_device():
    with pytest.raises(ValueError):
        release_cached_memory(-2)
