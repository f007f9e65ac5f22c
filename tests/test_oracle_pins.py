"""Pins the oracle (CPU restatement) before it is trusted as the checker.

* the reference's known answers (tests/test_gpu_pdhg.cpp:263-404, afiro
  -464.75314286 from tests/test_precision_ladder.cpp:353,419);
* the reference's own CPU check loops (tests/test_gpu_pdhg.cpp:147-167,
  tests/test_pdhg_kernel.cpp:76-103), restated here in numpy;
* the reference's own CPU solvers (oracle/_ref, compiled from its sources).
Golden trajectories recorded from the reference's GPU solver are checked in
test_golden_reference.py.
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN, SCALED, mps_model, primal_violation, random_csr
from pramaan_b200.generators import random_sparse_lp


@pytest.mark.parametrize("name", sorted(KNOWN))
def test_oracle_solves_reference_known_answers(name):
    model, obj, feas = KNOWN[name]
    r = oracle.solve_ref(model)
    assert r["status"] == 0, r
    assert abs(r["objective_value"] - obj) <= 1e-3 + 1e-4 * abs(obj)
    if feas:
        assert primal_violation(model, r["x"]) <= 1e-4


def test_oracle_scaled_terminates():
    r = oracle.solve_ref(SCALED)
    assert r["status"] in (0, 3)
    if r["status"] == 0:
        assert primal_violation(SCALED, r["x"]) <= 1e-3


def test_oracle_spmv_matches_reference_cpu_loops():
    rng = np.random.default_rng(3)
    for m, n in [(1, 1), (3, 7), (33, 65), (129, 40)]:
        rp, ci, v = random_csr(m, n, rng)
        x = (np.arange(n, dtype=np.float32) + 1) * np.float32(0.5)
        y = oracle.spmv_f32(rp, ci, v, x, m)
        ref = np.zeros(m, np.float32)
        for i in range(m):   # cpu_spmv, tests/test_gpu_pdhg.cpp:147-156
            for k in range(rp[i], rp[i + 1]):
                ref[i] = np.float32(ref[i] + np.float32(v[k] * x[ci[k]]))
        np.testing.assert_array_equal(y, ref)
        xt = (np.arange(m, dtype=np.float32) + 1) * np.float32(0.3)
        yt = oracle.spmv_t_f32(rp, ci, v, xt, m, n)
        reft = np.zeros(n, np.float32)
        for i in range(m):   # cpu_spmv_t, :158-167
            for k in range(rp[i], rp[i + 1]):
                reft[ci[k]] = np.float32(reft[ci[k]] + np.float32(v[k] * xt[i]))
        np.testing.assert_array_equal(yt, reft)


def test_oracle_step1_matches_reference_cpu_step():
    rng = np.random.default_rng(42)
    for _ in range(20):
        n, m = 150, 120
        x = rng.uniform(-10, 10, n).astype(np.float32)
        g = rng.uniform(-10, 10, n).astype(np.float32)
        y = rng.uniform(-10, 10, m).astype(np.float32)
        ax = rng.uniform(-10, 10, m).astype(np.float32)
        b = rng.uniform(-10, 10, m).astype(np.float32)
        tau, sig = np.float32(abs(rng.uniform(-10, 10))), np.float32(abs(rng.uniform(-10, 10)))
        xo, yo = oracle.step1(x, y, g, ax, b, tau, sig, use_fma=False)
        # cpu_pdhg_step (tests/test_pdhg_kernel.cpp:76-103)
        np.testing.assert_array_equal(xo, np.maximum(np.float32(0), x - tau * g))
        np.testing.assert_array_equal(yo, y + sig * (ax - b))


def test_oracle_step_sizes_follow_reference_rule():
    model = random_sparse_lp(50, 120, 4, seed=1)
    sig, tau = oracle.step_sizes(model)
    v = np.abs(model.values.astype(np.float32).astype(np.float64))
    rows = np.repeat(np.arange(model.numRows()), np.diff(model.row_ptr))
    rn = np.bincount(rows, weights=v, minlength=model.numRows())
    cn = np.bincount(model.col_idx, weights=v, minlength=model.numVars())
    exp_sig = np.where(rn > 1e-12, np.float32(0.95) / rn.astype(np.float32), np.float32(0.95))
    exp_tau = np.where(cn > 1e-12, np.float32(0.95) / cn.astype(np.float32), np.float32(0.95))
    np.testing.assert_allclose(sig, exp_sig.astype(np.float32), rtol=1e-6)
    np.testing.assert_allclose(tau, exp_tau.astype(np.float32), rtol=1e-6)


def test_oracle_residuals_match_numpy_restatement():
    model = random_sparse_lp(40, 100, 4, seed=2)
    rng = np.random.default_rng(0)
    x = rng.uniform(-0.5, 3, model.numVars()).astype(np.float32)
    y = rng.standard_normal(model.numRows()).astype(np.float32)
    tol = 1e-3
    pv, dv = oracle.residuals_ref(model, x, y, tol)
    xd = x.astype(np.float64)
    act = model.multiply(xd)
    p = max(np.max(np.maximum(model.row_lower - act, 0)), np.max(np.maximum(act - model.row_upper, 0)),
            np.max(np.maximum(model.var_lower - xd, 0)), np.max(np.maximum(xd - model.var_upper, 0)))
    rows = np.repeat(np.arange(model.numRows()), np.diff(model.row_ptr))
    aty = np.bincount(model.col_idx, weights=model.values.astype(np.float32).astype(np.float64) * y[rows],
                      minlength=model.numVars())
    c32 = model.obj_coeffs.astype(np.float32).astype(np.float64)
    rc = c32 + aty
    at_lb = xd <= model.var_lower + tol
    at_ub = xd >= model.var_upper - tol
    viol = np.where(~at_lb & ~at_ub, np.abs(rc),
                    np.where(at_lb & ~at_ub, np.maximum(0, -rc), np.where(at_ub & ~at_lb, np.maximum(0, rc), 0)))
    d = np.max(viol) / max(1.0, np.max(np.abs(c32)))
    assert pv == pytest.approx(p, rel=1e-12, abs=1e-300)
    assert dv == pytest.approx(d, rel=1e-12, abs=1e-300)


def test_oracle_certificate_math():
    model, obj, _ = KNOWN["wyndor"]
    c = oracle.certificate(model, np.array([2.0, 6.0]))
    assert c["objective"] == pytest.approx(36.0)
    assert c["primal_residual"] <= 0 + 1e-15 and c["bound_violation"] == 0.0
    c = oracle.certificate(model, np.array([5.0, 0.0]))
    assert c["primal_residual"] == pytest.approx(1.0) and c["bound_violation"] == 0.0


def test_oracle_rel_kkt_zero_at_constructed_optimum():
    # x0 feasible; (y0, s0) dual feasible; at the constructed pair the primal
    # and dual residuals vanish and the gap equals s0^T x0 (a sanity anchor).
    model, cert = random_sparse_lp(30, 80, 4, seed=5, return_certificate=True)
    k = oracle.rel_kkt(model, cert["x0"], -cert["y0"])
    assert k["primal"] < 1e-12
    assert k["dual"] < 1e-12
    assert k["pobj"] - k["dobj"] == pytest.approx(float(cert["s0"] @ cert["x0"]), rel=1e-9)


@pytest.mark.skipif(oracle.ref_cpu() is None, reason="oracle/_ref not built (needs the reference tree)")
def test_oracle_afiro_matches_reference_simplex():
    model = mps_model("afiro")
    cpu = oracle.ref_solve("simplex", model)
    assert cpu["status"] == 0
    assert cpu["objective_value"] == pytest.approx(-464.75314286, abs=1e-6)
    r = oracle.solve_ref(model, tol=1e-5, max_iterations=200000, check_frequency=500)
    assert r["status"] == 0
    assert abs(r["objective_value"] - cpu["objective_value"]) <= 1e-4


@pytest.mark.skipif(oracle.ref_cpu() is None, reason="oracle/_ref not built (needs the reference tree)")
def test_oracle_small_random_lp_matches_reference_simplex():
    model = random_sparse_lp(20, 60, 4, seed=7)
    cpu = oracle.ref_solve("simplex", model, max_iterations=100000)
    assert cpu["status"] == 0
    r = oracle.solve_ref(model, tol=1e-6, max_iterations=200000, check_frequency=100)
    assert r["status"] == 0
    assert abs(r["objective_value"] - cpu["objective_value"]) <= 1e-4 * (1 + abs(cpu["objective_value"]))


# ---- the numpy restatement of the adaptive mode (oracle/adaptive.py) ----------

def test_adaptive_restatement_rel_kkt_equals_c_oracle():
    from oracle import adaptive as ada
    rng = np.random.default_rng(11)
    for name in ("wyndor", "multi", "bounded"):
        model = KNOWN[name][0]
        x = rng.uniform(-1, 5, model.numVars())
        y = rng.uniform(-2, 2, model.numRows())
        mine = ada.rel_kkt(ada.problem(model), x, y)
        ref = oracle.rel_kkt(model, x, y)
        for a, b in (("rel_p", "primal"), ("rel_d", "dual"), ("rel_gap", "gap"), ("pobj", "pobj"),
                     ("dobj", "dobj")):
            assert mine[a] == pytest.approx(ref[b], rel=1e-12, abs=1e-14), (name, a)


@pytest.mark.parametrize("name", ["wyndor", "multi", "equality", "bounded"])
def test_adaptive_restatement_solves_known_answers(name):
    from oracle import adaptive as ada
    model, obj, _ = KNOWN[name]
    r = ada.solve(model, tol=1e-8, max_iterations=50000)
    assert r["status"] == "optimal"
    sgn = -1.0 if int(model.obj_sense) == 1 else 1.0
    assert sgn * r["kkt"]["pobj"] + model.obj_offset == pytest.approx(obj, rel=1e-7, abs=1e-7)
