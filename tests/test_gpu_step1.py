"""GPU parity of the Step-1 dense iteration (pramaan_launch_pdhg_iteration)
with the reference's test cases (tests/test_pdhg_kernel.cpp:129-241).

Two checks per case: bit-exact against the oracle's device form (the FMA
contraction nvcc applies to the reference kernel), and within the reference's
own tolerance (atol 1e-5, rtol 1e-4) against its CPU step (no FMA).
"""
import numpy as np
import pytest

import oracle
from pramaan_b200 import launch_pdhg_iteration

pytestmark = pytest.mark.gpu


def near(a, b, atol, rtol):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    assert a.shape == b.shape
    eq = a == b
    ok = eq | (np.isfinite(a) & np.isfinite(b) & (np.abs(a - b) <= atol + rtol * np.maximum(np.abs(a), np.abs(b))))
    assert ok.all(), np.nonzero(~ok)[0][:5]


def run_case(x, y, g, ax, b, tau, sigma):
    x = np.array(x, np.float32)
    y = np.array(y, np.float32)
    ex_fma = oracle.step1(x, y, g, ax, b, np.float32(tau), np.float32(sigma), use_fma=True)
    ex_cpu = oracle.step1(x, y, g, ax, b, np.float32(tau), np.float32(sigma), use_fma=False)
    launch_pdhg_iteration(x, y, g, ax, b, tau, sigma)
    np.testing.assert_array_equal(x, ex_fma[0])
    np.testing.assert_array_equal(y, ex_fma[1])
    near(ex_cpu[0], x, 1e-5, 1e-4)
    near(ex_cpu[1], y, 1e-5, 1e-4)


def test_primal_edge_cases():
    run_case([1, 1, 2, 1, 0, 5, 1, 1], [], [0.5, -0.5, 2, 3, 1, 0, 1e5, -1e5], [], [], 1.0, 1.0)


@pytest.mark.parametrize("sigma", [1.0, 0.0])
def test_dual_edge_cases(sigma):
    run_case([], [0, 0, 0, 5, 0, 2, 1e5, 1e-5, -2], [], [1, -1, 1, 2, 1, 0, -1e5, 1e-5, 0],
             [0, 0, 1, 2, 0, 0, 0, 0, 0], 1.0, sigma)


@pytest.mark.parametrize("d", [0, 1, 2, 3, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 1024, 1025])
def test_dimension_coverage(d):
    run_case(np.ones(d), np.ones(d), np.full(d, 0.5), np.full(d, 0.5), np.zeros(d), 1.0, 1.0)


def test_matrix_free_shapes():
    run_case([1], [1], [1], [1], [1], 1.0, 1.0)
    run_case([], [1], [], [1], [1], 1.0, 1.0)
    run_case([1], [], [1], [], [], 1.0, 1.0)
    run_case([], [], [], [], [], 1.0, 1.0)


def test_randomized():
    rng = np.random.default_rng(42)
    for it in range(50):
        n, m = 150, 120
        x = rng.uniform(-10, 10, n).astype(np.float32)
        x[::7] = 0
        g = rng.uniform(-10, 10, n).astype(np.float32)
        y = rng.uniform(-10, 10, m).astype(np.float32)
        ax = rng.uniform(-10, 10, m).astype(np.float32)
        b = rng.uniform(-10, 10, m).astype(np.float32)
        b[::7] = 0
        run_case(x, y, g, ax, b, abs(rng.uniform(-10, 10)), abs(rng.uniform(-10, 10)))


def test_numerical_stress():
    run_case([1e-10, 1e10, 1e-38, 1.0, 0.0, -0.0], [1e-10, 1e10, 1e-38, -1e-38],
             [1e-10, -1e10, -1e-38, 1.0, 1e-38, -1e-38], [1e-10, 1e10, 1e-38, -1e-38],
             [1e-10, 1e10, 1e-38, -1e-38], 1.0, 1.0)


def test_repeated_execution():
    x = np.ones(1000, np.float32)
    y = np.ones(1000, np.float32)
    g = np.full(1000, 0.1, np.float32)
    ax = np.full(1000, 0.1, np.float32)
    b = np.zeros(1000, np.float32)
    cx, cy = x.copy(), y.copy()
    for _ in range(50):
        launch_pdhg_iteration(x, y, g, ax, b, 1.0, 1.0)
        cx, cy = oracle.step1(cx, cy, g, ax, b, np.float32(1), np.float32(1), use_fma=False)
    near(cx, x, 1e-3, 1e-3)
    near(cy, y, 1e-3, 1e-3)
