"""GPU tests of the warm-start network (pramaan_gnn_*) and of warm-started
batched solves (pramaan_pdhg_solve_batch_warm).

The network has no reference counterpart; its checker is the NumPy
restatement oracle/gnn.py in BF16 mode (the same rounding points).  Summation
orders differ (tensor-core accumulation, per-row gathers), so a BF16 rounding
can land on the other side of a tie; the tolerances are relative Frobenius
errors per activation or parameter block: 1e-2 for activations, 3e-2 for
gradient blocks, 1e-3 for the loss.
"""
import numpy as np
import pytest

from lp_cases import KNOWN
from oracle import gnn as og
from pramaan_b200 import PdhgOptions, SolveStatus, solve_batch
from pramaan_b200.generators import (random_sparse_lp, rolling_horizon_batch, rolling_horizon_lp,
                                    rolling_horizon_tail_mask)
from pramaan_b200.gnn import WarmStart, WarmStartNet, training_targets, warm_solve_batch
from pramaan_b200.pdhg import ALGO_ADAPTIVE

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def split_trace(g, flat):
    out, off = {}, 0
    for name, shape in og.trace_layout(g):
        size = int(np.prod(shape))
        out[name] = flat[off:off + size].reshape(shape)
        off += size
    assert off == len(flat)
    return out


def small_models():
    return [rolling_horizon_lp(30, 7, seed=1), random_sparse_lp(50, 130, 3, seed=2), KNOWN["wyndor"][0],
            rolling_horizon_lp(13, 3, seed=3)]


def targets_for(models, seed=0):
    rng = np.random.default_rng(seed)
    return [WarmStart(rng.uniform(0, 20, md.numVars()), rng.normal(0, 2, md.numRows()),
                      float(np.exp(rng.normal(0, 1)))) for md in models]


def check_trace(models, seed):
    net = WarmStartNet(seed=seed)
    net.params = og.init_params(seed).astype(np.float32)   # non-zero heads
    p = net.params
    G = net.graph(models)
    tr = split_trace(og.Graph(models), net.trace(G))
    a = og.forward(p, og.Graph(models), exact=False)
    for l in range(og.LAYERS):
        assert rel(tr[f"xc{l}"], a["xc"][l]) < 1e-2, ("xc", l)
        assert rel(tr[f"xv{l}"], a["xv"][l]) < 1e-2, ("xv", l)
    for name in ("hc3", "hv3", "xhat", "yhat", "pooled", "rho"):
        assert rel(tr[name], a[name]) < 1e-2, name
    # the layer outputs are BF16 values and non-negative
    assert np.all(tr["hv3"] >= 0) and np.all(tr["hv3"].view(np.uint32) & 0xFFFF == 0)


def test_forward_matches_oracle():
    check_trace(small_models(), seed=1)


def test_forward_matches_oracle_over_many_tiles():
    # > 2 x 148 x 128 variable rows: every block of the dense kernels loops over several tiles
    models = rolling_horizon_batch(6, seed=5, T_range=(100, 120), P_range=(20, 25))
    assert sum(md.numVars() for md in models) > 2 * 148 * 128
    check_trace(models, seed=2)


def blocks():
    out = {"vin": (og.VIN_W, og.CIN_W), "cin": (og.CIN_W, og.LAYER0)}
    for l in range(og.LAYERS):
        for side, nm in ((0, "c"), (1, "v")):
            out[f"W{nm}{l}"] = (og.layer_w(l, side), og.layer_b(l, side))
            out[f"b{nm}{l}"] = (og.layer_b(l, side), og.layer_b(l, side) + 64)
    out["heads"] = (og.HEAD_X, og.COUNT)
    return out


@pytest.mark.parametrize("big", [False, True])
def test_gradients_match_oracle(big):
    models = (rolling_horizon_batch(6, seed=7, T_range=(100, 120), P_range=(20, 25)) if big
              else small_models())
    tg = targets_for(models, seed=3)
    net = WarmStartNet(seed=4)
    net.params = og.init_params(4).astype(np.float32)      # non-zero heads: every block has a gradient
    p = net.params
    loss, grad = net.gradients(net.graph(models, tg))
    oloss, ograd = og.loss_and_grad(p, og.Graph(models, tg), exact=False)
    assert loss == pytest.approx(oloss, rel=1e-3)
    for name, (b, e) in blocks().items():
        assert rel(grad[b:e], ograd[b:e]) < 3e-2, name
    assert rel(grad, ograd) < 1e-2


def test_gradients_are_deterministic():
    models = small_models()
    tg = targets_for(models, seed=5)
    net = WarmStartNet(seed=6)
    net.params = og.init_params(6).astype(np.float32)
    g = net.graph(models, tg)
    l1, g1 = net.gradients(g)
    l2, g2 = net.gradients(g)
    assert l1 == l2 and np.array_equal(g1, g2)


def test_params_roundtrip_and_seed():
    a, b = WarmStartNet(seed=11), WarmStartNet(seed=11)
    assert np.array_equal(a.params, b.params)
    # heads start at zero: the untrained network returns its hint unchanged
    assert not a.params[og.HEAD_X:].any()
    p = og.init_params(3).astype(np.float32)
    a.params = p
    assert np.array_equal(a.params, p)


def test_training_fits_solved_targets():
    models = rolling_horizon_batch(12, seed=8, T_range=(24, 36), P_range=(5, 8))
    res = solve_batch(models, PdhgOptions(tolerance=1e-4, max_iterations=200000, check_frequency=64,
                                          algorithm=ALGO_ADAPTIVE))
    assert all(r.status == SolveStatus.kOptimal for r in res)
    net = WarmStartNet(seed=0)
    graphs = [net.graph(models[i:i + 4], training_targets(res[i:i + 4])) for i in range(0, 12, 4)]
    hist = net.fit(graphs, epochs=120, lr=3e-3)
    assert hist[-1] < 0.75 * hist[0], hist
    # the trained network's loss, recomputed by the oracle from its parameters
    g = graphs[0]
    loss, _ = net.gradients(g)
    oloss, _ = og.loss_and_grad(net.params, og.Graph(models[:4], training_targets(res[:4])), exact=False)
    assert loss == pytest.approx(oloss, rel=1e-3)


def test_untrained_network_returns_the_hint():
    models = small_models()
    rng = np.random.default_rng(2)
    hints = [WarmStart(rng.uniform(0, 5, md.numVars()), rng.normal(0, 1, md.numRows()), 0.0) for md in models]
    net = WarmStartNet(seed=3)
    pred = net.predict(models, hints=hints)
    for md, h, p in zip(models, hints, pred):
        lo, hi = md.var_lower, md.var_upper
        np.testing.assert_allclose(p.x, np.clip(h.x, lo, hi), rtol=1e-6, atol=1e-6 * np.abs(h.x).max())
        np.testing.assert_allclose(p.y, h.y, rtol=1e-6, atol=1e-6 * np.abs(h.y).max())
    # and with hints, the gradients still match the oracle
    tg = targets_for(models, seed=4)
    net.params = og.init_params(5).astype(np.float32)
    loss, grad = net.gradients(net.graph(models, tg, hints))
    oloss, ograd = og.loss_and_grad(net.params, og.Graph(models, tg, hints), exact=False)
    assert loss == pytest.approx(oloss, rel=1e-3)
    assert rel(grad, ograd) < 1e-2


def opts(tol=1e-6, it=300000):
    return PdhgOptions(tolerance=tol, max_iterations=it, check_frequency=64, algorithm=ALGO_ADAPTIVE)


def test_warm_start_none_is_the_cold_start():
    models = rolling_horizon_batch(4, seed=9, T_range=(24, 30), P_range=(5, 6))
    a = solve_batch(models, opts())
    b = solve_batch(models, opts(), warm=[None] * 4)
    for ra, rb in zip(a, b):
        assert ra.iterations == rb.iterations and np.array_equal(ra.x, rb.x)


def test_warm_start_from_the_solution_stops_early():
    models = rolling_horizon_batch(4, seed=10, T_range=(24, 30), P_range=(5, 6)) + [KNOWN["wyndor"][0]]
    cold = solve_batch(models, opts())
    warm = solve_batch(models, opts(), warm=training_targets(cold))
    for c, w in zip(cold, warm):
        assert c.status == w.status == SolveStatus.kOptimal
        assert w.iterations <= 64 < c.iterations
        assert w.objective_value == pytest.approx(c.objective_value, rel=1e-5, abs=1e-5)


def test_warm_solve_falls_back_to_cold():
    # an untrained network's point may not converge within a tiny budget: the
    # fallback re-solves those LPs cold with a full budget
    models = rolling_horizon_batch(4, seed=12, T_range=(24, 30), P_range=(5, 6))
    net = WarmStartNet(seed=1)
    res, info = warm_solve_batch(models, net, opts(it=128), fallback_iterations=300000)
    assert info.fallbacks >= 1
    assert all(r.status == SolveStatus.kOptimal for r in res)


def _stream_set(seeds, count, T_range, P_range):
    from pramaan_b200.generators import rolling_horizon_stream
    ms, first = [], []
    for s in seeds:
        ms += rolling_horizon_stream(count, seed=s, T_range=T_range, P_range=P_range)
        first += [True] + [False] * (count - 1)
    return ms, first


def _hints(ms, first, res):
    from pramaan_b200.generators import rolling_horizon_shift
    out = []
    for i, md in enumerate(ms):
        if first[i]:
            out.append(None)
            continue
        PT = md.numVars() // 3
        T = md.numRows() - PT
        xs, ys = rolling_horizon_shift(res[i - 1].x, res[i - 1].y, T, PT // T)
        out.append(WarmStart(xs, ys, 0.0))
    return out


def test_learned_warm_start_saves_iterations_on_a_stream():
    """Train on solved windows of some streams, then solve held-out streams:
    the certified learned warm start (network refining the previous window's
    shifted solution, the certificate choosing each LP's start) needs fewer
    PDHG iterations in total than cold starts, and every answer meets the
    tolerance on the FP64 certificate."""
    from pramaan_b200.certificate import certify_batch
    o = opts()
    TR, PR = (24, 48), (5, 10)
    train, ftr = _stream_set(range(3000, 3080), 5, TR, PR)
    ev, fev = _stream_set(range(3900, 3903), 12, TR, PR)
    rtr = solve_batch(train, o)
    cold = solve_batch(ev, o)
    assert all(r.status == SolveStatus.kOptimal for r in rtr + cold)
    htr, hev = _hints(train, ftr, rtr), _hints(ev, fev, cold)
    idx = [i for i in range(len(train)) if htr[i] is not None]
    net = WarmStartNet(seed=0)
    graphs = [net.graph([train[i] for i in idx[k:k + 16]], training_targets([rtr[i] for i in idx[k:k + 16]]),
                        hints=[htr[i] for i in idx[k:k + 16]]) for k in range(0, len(idx), 16)]
    net.fit(graphs, epochs=30, lr=1e-3, lr_decay=0.97)
    res, info = warm_solve_batch(ev, net, o, hints=hev)
    cold_total = sum(r.iterations for r in cold)
    warm_total = sum(info.warm_iterations)
    print(f"learned warm start: {warm_total} iterations vs {cold_total} cold "
          f"({warm_total / cold_total:.3f}); starts {dict((c, info.choices.count(c)) for c in set(info.choices))}")
    assert warm_total < 0.9 * cold_total
    cert = certify_batch(ev, [[WarmStart(r.x, r.y) for r in res]])[0]
    for r, c in zip(res, cert):
        assert r.status == SolveStatus.kOptimal and c.kkt <= 1e-6 * 1.0001


def test_learned_start_measured_against_the_hint_it_refines():
    """What the trained network adds over the method without it.  The method
    without it starts each window from the previous window's shifted solution
    (the hint).  The certified learned pipeline lets the FP64 certificate
    choose, after a 64-iteration probe from each candidate, between the
    network's refinement of the hint, the hint, their midpoint and the cold
    start.  On held-out streams both are measured in total PDHG iterations,
    the learned pipeline's probes included.  The network's refinement is not
    a reliable gain over the hint it refines (on the benchmark stream it
    needs 5 % more iterations), and neither is the network confined to the
    last periods of each window (the hint elsewhere): within a few per cent
    of the hint either way on held-out streams.  So what is asserted is that
    both learned pipelines stay close to the hint, that all beat cold starts,
    and that every answer is certified."""
    from pramaan_b200.certificate import certify_batch
    from pramaan_b200.train_warm_start import DEFAULT_OUT
    o = opts()
    ev, fev = _stream_set(range(3950, 3956), 6, (24, 96), (5, 20))
    cold = solve_batch(ev, o)
    assert all(r.status == SolveStatus.kOptimal for r in cold)
    hev = _hints(ev, fev, cold)
    net = WarmStartNet(seed=0)
    net.load(DEFAULT_OUT)
    hint = solve_batch(ev, o, warm=hev)
    res, info = warm_solve_batch(ev, net, o, hints=hev, probe_iterations=64)
    cold_total = sum(r.iterations for r in cold)
    hint_total = sum(r.iterations for r in hint)
    learned_total = sum(info.warm_iterations) + info.probe_iterations
    # the network on the last four periods of each window only, the hint elsewhere, no selection
    masks = []
    for md, h in zip(ev, hev):
        T = md.numRows() - md.numVars() // 3
        masks.append(None if h is None else rolling_horizon_tail_mask(T, md.numVars() // (3 * T), 4))
    res_t, info_t = warm_solve_batch(ev, net, o, hints=hev, refine_masks=masks, select=False)
    tail_total = sum(info_t.warm_iterations)
    print(f"iterations: cold {cold_total}, hint {hint_total} ({hint_total / cold_total:.3f}), learned "
          f"{learned_total} ({learned_total / cold_total:.3f}, {learned_total / hint_total:.3f} of hint); "
          f"starts {dict((c, info.choices.count(c)) for c in set(info.choices))}; network on the last 4 periods "
          f"{tail_total} ({tail_total / hint_total:.3f} of hint)")
    assert hint_total < cold_total and learned_total < cold_total and tail_total < cold_total
    assert learned_total <= 1.15 * hint_total and tail_total <= 1.15 * hint_total
    cert = certify_batch(ev, [[WarmStart(r.x, r.y) for r in res], [WarmStart(r.x, r.y) for r in res_t]])
    for rr, cc in ((res, cert[0]), (res_t, cert[1])):
        for r, c in zip(rr, cc):
            assert r.status == SolveStatus.kOptimal and c.kkt <= 1e-6 * 1.0001
