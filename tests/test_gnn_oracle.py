"""CPU tests of the warm-start network's NumPy restatement (oracle/gnn.py).

The oracle is the checker of the GPU network, so its backward pass is pinned
here against central finite differences of its own loss in exact (float64,
unrounded) arithmetic, and its BF16 rounding and graph features against
values worked out by hand.
"""
import numpy as np
import pytest

from lp_cases import KNOWN
from oracle import gnn as og
from pramaan_b200.generators import random_sparse_lp, rolling_horizon_lp, rolling_horizon_stream
from pramaan_b200.gnn import WarmStart
from pramaan_b200.pdhg import ModelIR


def _targets(models, seed=0):
    rng = np.random.default_rng(seed)
    return [WarmStart(rng.uniform(0, 3, md.numVars()), rng.normal(0, 1, md.numRows()),
                      float(np.exp(rng.normal(0, 1)))) for md in models]


def test_bf16_rounding():
    v = np.array([1.0, 1.00390625, 1.01171875, 1.005859375, -2.5, 3.0e-3, 0.0, 65504.0], np.float32)
    r = og.bf16(v)
    # 1.00390625 = 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa -> 1.0
    assert r[0] == 1.0 and r[1] == 1.0
    # 1 + 3*2^-8 is a tie between 1 + 2^-7 (odd) and 1 + 2^-6 (even) -> 1 + 2^-6
    assert r[2] == np.float32(1.015625)
    assert r[3] == np.float32(1.0078125)
    assert r[4] == -2.5 and r[6] == 0.0
    assert abs(r[5] - 3.0e-3) <= 3.0e-3 * 2 ** -8
    assert r[7] == 65536.0
    # every output has an all-zero low half
    assert np.all(r.view(np.uint32) & 0xFFFF == 0)


def test_features_by_hand():
    wyndor = KNOWN["wyndor"][0]        # max 3x1 + 5x2; x1 <= 4, 2x2 <= 12, 3x1 + 2x2 <= 18
    g = og.Graph([wyndor])
    sa = np.sqrt(np.mean(np.asarray(wyndor.values) ** 2))
    assert g.s_a[0] == pytest.approx(sa)
    b = np.array([v for v in wyndor.row_upper if v < 1e29] + [v for v in wyndor.row_lower if v > -1e29])
    assert g.s_b[0] == pytest.approx(np.sqrt(np.mean(b ** 2)))
    # costs negated for the maximisation
    assert g.fv[0, 0] == pytest.approx(-3.0 / g.s_c[0], rel=1e-6)
    assert g.fv[:, 7].tolist() == [0.0, 0.0] and g.fv[:, 8].tolist() == [0.0, 0.0]   # no hint
    # x1 appears in two rows: log(3)/4
    assert g.fv[0, 5] == pytest.approx(np.log(3.0) / 4, rel=1e-6)
    # row 2: 3x1 + 2x2 <= 18: mean |A| / s_a
    assert g.fc[2, 6] == pytest.approx(2.5 / sa, rel=1e-6)
    assert g.fc[2, 2] == 1.0 and g.fc[2, 4] == pytest.approx(min(10, 18 / g.s_b[0]), rel=1e-6)


@pytest.mark.parametrize("seed", [0, 1])
def test_exact_gradient_matches_finite_differences(seed):
    models = [rolling_horizon_lp(4, 2, seed=seed), random_sparse_lp(6, 12, 2, seed=seed), KNOWN["wyndor"][0]]
    g = og.Graph(models, _targets(models, seed))
    p = og.init_params(seed)
    # move the biases off zero so that every ReLU has a defined slope
    rng = np.random.default_rng(seed + 10)
    p += rng.normal(0, 0.05, og.COUNT)
    loss, grad = og.loss_and_grad(p, g, exact=True)
    assert np.isfinite(loss) and loss > 0
    idx = np.concatenate([
        rng.choice(og.COUNT, 60, replace=False),
        [og.HEAD_X + 64, og.HEAD_Y + 64, og.HEAD_W + 128, og.VIN_B, og.CIN_B],
        [og.layer_w(0, 0) + 5, og.layer_w(2, 1) + 100, og.layer_b(1, 0) + 3],
    ])
    h = 1e-6
    for i in idx:
        e = np.zeros(og.COUNT)
        e[i] = h
        lp, _ = og.loss_and_grad(p + e, g, exact=True, grad=False)
        lm, _ = og.loss_and_grad(p - e, g, exact=True, grad=False)
        fd = (lp - lm) / (2 * h)
        assert grad[i] == pytest.approx(fd, rel=1e-4, abs=1e-7), (int(i), grad[i], fd)


def test_hints_enter_features_and_heads():
    models = [rolling_horizon_lp(3, 2, seed=5), KNOWN["wyndor"][0]]
    rng = np.random.default_rng(1)
    hints = [WarmStart(rng.uniform(0, 50, models[0].numVars()), None, 0.0),
             WarmStart(None, rng.normal(0, 3, 3), 0.0)]
    g0, g1 = og.Graph(models), og.Graph(models, hints=hints)
    p = og.init_params(2)
    a0, a1 = og.forward(p, g0, exact=True), og.forward(p, g1, exact=True)
    n0 = models[0].numVars()
    assert g1.fv[:n0, 7].all() and not g1.fv[n0:, 7].any()
    assert g1.fc[models[0].numRows():, 7].all() and not g1.fc[:models[0].numRows(), 7].any()
    np.testing.assert_allclose(g1.fv[:n0, 8], np.clip(hints[0].x * g1.s_a[0] / g1.s_b[0], -10, 10), rtol=1e-6)
    # the heads add the scaled hint to the network's correction
    assert not np.allclose(a0["xhat"][:n0], a1["xhat"][:n0])
    # gradients stay exact with hints
    tg = _targets(models, 3)
    g2 = og.Graph(models, tg, hints)
    loss, grad = og.loss_and_grad(p, g2, exact=True)
    e = np.zeros(og.COUNT)
    i = og.VIN_W + 8             # the weight of the hint-value feature
    e[i] = 1e-6
    fd = (og.loss_and_grad(p + e, g2, exact=True, grad=False)[0] - og.loss_and_grad(p - e, g2, exact=True, grad=False)[0]) / 2e-6
    assert grad[i] == pytest.approx(fd, rel=1e-4, abs=1e-7)


def test_loss_is_zero_at_the_prediction():
    models = [rolling_horizon_lp(3, 2, seed=4)]
    g = og.Graph(models)
    p = og.init_params(3)
    a = og.forward(p, g, exact=True)
    q = 0
    sa, sb, sc = g.s_a[q], g.s_b[q], g.s_c[q]
    t = WarmStart(a["xhat"] * sb / sa, a["yhat"] * sc / sa, float(g.omega_ref[q] * np.exp(a["rho"][q])))
    g2 = og.Graph(models, [t])
    loss, grad = og.loss_and_grad(p, g2, exact=True)
    assert loss == pytest.approx(0.0, abs=1e-20)
    assert np.max(np.abs(grad)) == pytest.approx(0.0, abs=1e-12)


def test_graph_skips_empty_lps_and_handles_row_free_lps():
    empty = ModelIR([], [0, 0], [], [], [1.0], [2.0], [], [], 0, 0.0)
    free = ModelIR([1.0, -2.0], [0], [], [], [], [], [0.0, 0.0], [1.0, 1.0], 0, 0.0)
    wy = KNOWN["wyndor"][0]
    g = og.Graph([empty, free, wy], [None, WarmStart(np.ones(2), np.zeros(0), 1.0),
                                     WarmStart(np.ones(2), np.ones(3), 2.0)])
    assert g.index == [1, 2] and g.K == 2 and g.m == 3 and g.n == 4
    loss, grad = og.loss_and_grad(og.init_params(0), g, exact=True)
    assert np.isfinite(loss) and np.all(np.isfinite(grad))


def test_stream_windows_shift_by_one_period():
    s = rolling_horizon_stream(4, seed=2, T=6, P=3)
    T, P = 6, 3
    for a, b in zip(s, s[1:]):
        da = a.row_lower[:P * T].reshape(P, T)
        db = b.row_lower[:P * T].reshape(P, T)
        np.testing.assert_array_equal(da[:, 1:], db[:, :-1])
        ca = a.obj_coeffs.reshape(3, P, T)
        cb = b.obj_coeffs.reshape(3, P, T)
        np.testing.assert_array_equal(ca[:, :, 1:], cb[:, :, :-1])
        np.testing.assert_array_equal(a.row_upper[P * T + 1:], b.row_upper[P * T:-1])
