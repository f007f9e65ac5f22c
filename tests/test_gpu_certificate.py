"""GPU tests of the FP64 certificates (pramaan_certify_batch).

The checker is the oracle's FP64 restatement of the reference certificate
(src/certificate/certificate.cpp:23-107, oracle.certificate) and its relative
KKT (oracle.rel_kkt).  Both sides compute in FP64; the device sums in another
order and reads the matrix as FP32 hi + lo (exact to 2^-48 of each value), so
the comparison is at 1e-9 relative.
"""
import numpy as np
import pytest

import oracle
from lp_cases import KNOWN
from pramaan_b200 import PdhgOptions, SolveStatus, solve_batch
from pramaan_b200.certificate import certify_batch
from pramaan_b200.generators import ill_conditioned_lp, random_sparse_lp, rolling_horizon_batch
from pramaan_b200.gnn import WarmStart
from pramaan_b200.pdhg import ALGO_ADAPTIVE

pytestmark = pytest.mark.gpu


def models():
    out = [KNOWN[n][0] for n in ("wyndor", "multi", "bounded", "equality", "one_var", "zero_obj", "sparse_zeros")]
    out += [random_sparse_lp(60, 180, 4, seed=s) for s in range(3)]
    out += rolling_horizon_batch(3, seed=4, T_range=(24, 40), P_range=(5, 8))
    out.append(ill_conditioned_lp(300, 800, 4, seed=5, scale_exp=2))
    return out


def close(a, b, rtol=1e-9, atol=1e-12):
    return abs(a - b) <= atol + rtol * max(abs(a), abs(b))


def check(md, cert, x, y):
    ref = oracle.certificate(md, x)
    kk = oracle.rel_kkt(md, x, y)
    assert close(cert.objective_value, ref["objective"], atol=1e-9), (cert.objective_value, ref["objective"])
    assert close(cert.primal_residual, max(ref["primal_residual"], 0.0), atol=1e-9)
    assert close(cert.bound_violation, max(ref["bound_violation"], 0.0), atol=1e-9)
    for mine, theirs in ((cert.rel_primal, kk["primal"]), (cert.rel_dual, kk["dual"]), (cert.rel_gap, kk["gap"]),
                         (cert.primal_objective, kk["pobj"]), (cert.dual_objective, kk["dobj"])):
        assert close(mine, theirs, atol=1e-10), (mine, theirs)
    assert cert.kkt == max(cert.rel_primal, cert.rel_dual, cert.rel_gap)


def test_random_points_match_the_oracle():
    ms = models()
    rng = np.random.default_rng(0)
    pts = [WarmStart(rng.normal(0, 3, md.numVars()), rng.normal(0, 2, md.numRows())) for md in ms]
    cert = certify_batch(ms, [pts])[0]
    for md, c, p in zip(ms, cert, pts):
        check(md, c, p.x, p.y)


def test_cold_start_and_several_point_sets():
    ms = models()
    rng = np.random.default_rng(1)
    a = [WarmStart(rng.uniform(0, 2, md.numVars()), None) for md in ms]
    b = [WarmStart(rng.uniform(-1, 1, md.numVars()), rng.normal(0, 1, md.numRows())) for md in ms]
    both = certify_batch(ms, [a, b, [None] * len(ms)])
    alone = certify_batch(ms, [b])[0]
    for md, ca, cb, cc, cb1, pa, pb in zip(ms, both[0], both[1], both[2], alone, a, b):
        check(md, ca, pa.x, np.zeros(md.numRows()))
        check(md, cb, pb.x, pb.y)
        assert cb == cb1          # packing once for many point sets changes nothing
        x0 = np.clip(np.zeros(md.numVars()), md.var_lower, md.var_upper)
        check(md, cc, x0, np.zeros(md.numRows()))


def test_solutions_certify_at_the_solver_tolerance():
    ms = models()
    res = solve_batch(ms, PdhgOptions(tolerance=1e-8, max_iterations=400000, check_frequency=64,
                                      algorithm=ALGO_ADAPTIVE))
    cert = certify_batch(ms, [[WarmStart(r.x, r.y) for r in res]])[0]
    for md, r, c in zip(ms, res, cert):
        assert r.status == SolveStatus.kOptimal
        assert c.kkt <= 1e-8 * 1.0001
        assert c.rel_primal == pytest.approx(r.rel_primal, rel=1e-6, abs=1e-14)
        assert c.objective_value == pytest.approx(r.objective_value, rel=1e-12, abs=1e-12)


def test_empty_and_row_free_lps():
    from pramaan_b200.pdhg import ModelIR
    empty = ModelIR([], [0, 0], [], [], [1.0], [2.0], [], [], 0, 3.0)
    free = ModelIR([1.0, -2.0], [0], [], [], [], [], [0.0, 0.0], [1.0, 1.0], 0, 0.5)
    c = certify_batch([empty, free], [[WarmStart(np.zeros(0), np.array([0.5])), WarmStart(np.array([2.0, 0.5]), None)]])[0]
    assert c[0].objective_value == 3.0 and c[0].primal_residual == 1.0   # row 0 <= 0*x: 0 < 1
    assert c[1].objective_value == pytest.approx(0.5 + 2.0 - 1.0)
    assert c[1].bound_violation == pytest.approx(1.0)
