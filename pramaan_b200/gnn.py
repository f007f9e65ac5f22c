"""Learned warm start for the batched PDHG: the graph network and its use.

``WarmStartNet`` wraps the network of libpramaan_b200 (pramaan_gnn_*): a
bipartite constraint-variable graph network with BF16 weights whose forward
and backward passes are hand-written sm_100a kernels (tensor-core dense
layers).  ``warm_solve_batch`` is the pipeline: predict (x, y, omega) for every
LP, solve the batch from those points, and re-solve cold any LP whose warm
solve did not reach the tolerance — plain cold-start PDHG is the fallback, and
every answer is judged by the same relative-KKT certificate as a cold solve.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .pdhg import ModelIR, PdhgOptions, SolveResult, SolveStatus, _f64, _ptr, solve_batch


@dataclass
class WarmStart:
    """A starting point for one LP (pramaan_warm_start)."""
    x: np.ndarray | None = None
    y: np.ndarray | None = None
    primal_weight: float = 0.0

    @staticmethod
    def from_result(r: SolveResult) -> "WarmStart":
        return WarmStart(np.asarray(r.x, np.float64), np.asarray(r.y, np.float64), float(r.primal_weight))


def _warm_array(models, points, required: bool):
    k = len(models)
    arr = (L.CWarmStart * max(k, 1))()
    keep = []
    for i, w in enumerate(points):
        if w is None:
            if required:
                raise ValueError("every LP needs a target point")
            arr[i].x, arr[i].y, arr[i].primal_weight = None, None, 0.0
            continue
        if required and w.x is None:
            raise ValueError("every target needs x")
        x = None if w.x is None else _f64(w.x)
        y = None if w.y is None else _f64(w.y)
        if x is not None and len(x) != models[i].numVars():
            raise ValueError("point x has the wrong length")
        if y is not None and len(y) != models[i].numRows():
            raise ValueError("point y has the wrong length")
        keep.extend([x, y])
        arr[i].x, arr[i].y, arr[i].primal_weight = _ptr(x), _ptr(y), float(w.primal_weight or 0.0)
    return arr, keep


class GnnGraph:
    """A batch of LPs packed for the network on one device (pramaan_gnn_graph)."""

    def __init__(self, models: list[ModelIR], targets: list[WarmStart] | None = None, device: int = 0,
                 hints: list[WarmStart | None] | None = None):
        self.models = list(models)
        self.device = device
        k = len(self.models)
        lps = (L.CLp * max(k, 1))()
        for i, md in enumerate(self.models):
            lps[i] = md.c_struct()
        tptr, hptr, keep = None, None, []
        if targets is not None:
            if len(targets) != k:
                raise ValueError("one target per model")
            tptr, kt = _warm_array(self.models, targets, True)
            keep += kt
        if hints is not None:
            if len(hints) != k:
                raise ValueError("one hint (or None) per model")
            hptr, kh = _warm_array(self.models, hints, False)
            keep += kh
        h = C.c_void_p()
        L.check(L.lib().pramaan_gnn_graph_create(lps, k, hptr, tptr, device, C.byref(h)))
        self.handle = h
        del keep

    def close(self):
        if getattr(self, "handle", None):
            L.lib().pramaan_gnn_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def trace_size(self) -> int:
        return int(L.lib().pramaan_gnn_trace_size(self.handle))


class WarmStartNet:
    """The warm-start network on one device (pramaan_gnn)."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.device = device
        h = C.c_void_p()
        L.check(L.lib().pramaan_gnn_create(device, C.c_uint64(seed), C.byref(h)))
        self.handle = h

    @staticmethod
    def num_params() -> int:
        return int(L.lib().pramaan_gnn_num_params())

    def close(self):
        if getattr(self, "handle", None):
            L.lib().pramaan_gnn_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()

    # ---- parameters ----
    @property
    def params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), np.float32)
        L.check(L.lib().pramaan_gnn_get_params(self.handle, _ptr(p)))
        return p

    @params.setter
    def params(self, value):
        p = np.ascontiguousarray(np.asarray(value, np.float32))
        if p.shape != (self.num_params(),):
            raise ValueError(f"expected {self.num_params()} parameters")
        L.check(L.lib().pramaan_gnn_set_params(self.handle, _ptr(p)))

    def save(self, path) -> None:
        np.savez(path, params=self.params)

    def load(self, path) -> None:
        self.params = np.load(path)["params"]

    # ---- graphs ----
    def graph(self, models, targets=None, hints=None) -> GnnGraph:
        return GnnGraph(models, targets, self.device, hints)

    # ---- inference / training ----
    def predict(self, models_or_graph, hints=None) -> list[WarmStart | None]:
        """Predicted starting point of every LP (None for LPs without variables)."""
        g = (models_or_graph if isinstance(models_or_graph, GnnGraph)
             else self.graph(models_or_graph, hints=hints))
        models = g.models
        k = len(models)
        xs = [np.zeros(md.numVars()) for md in models]
        ys = [np.zeros(md.numRows()) for md in models]
        xp = (C.c_void_p * max(k, 1))(*[_ptr(x) for x in xs])
        yp = (C.c_void_p * max(k, 1))(*[_ptr(y) for y in ys])
        om = np.zeros(max(k, 1))
        L.check(L.lib().pramaan_gnn_predict(self.handle, g.handle, xp, yp, _ptr(om)))
        return [WarmStart(xs[i], ys[i], float(om[i])) if models[i].numVars() else None for i in range(k)]

    def gradients(self, g: GnnGraph) -> tuple[float, np.ndarray]:
        grad = np.zeros(self.num_params(), np.float32)
        loss = C.c_double()
        L.check(L.lib().pramaan_gnn_gradients(self.handle, g.handle, _ptr(grad), C.byref(loss)))
        return loss.value, grad

    def train_step(self, g: GnnGraph, lr: float = 1e-3) -> float:
        loss = C.c_double()
        L.check(L.lib().pramaan_gnn_train_step(self.handle, g.handle, C.c_float(lr), C.byref(loss)))
        return loss.value

    def trace(self, g: GnnGraph) -> np.ndarray:
        out = np.zeros(max(g.trace_size, 1), np.float32)
        L.check(L.lib().pramaan_gnn_forward_trace(self.handle, g.handle, _ptr(out)))
        return out[:g.trace_size]

    def fit(self, graphs: list[GnnGraph], epochs: int = 10, lr: float = 1e-3, lr_decay: float = 1.0,
            seed: int = 0) -> list[float]:
        """Adam over the given mini-batch graphs; returns the mean loss of each epoch."""
        rng = np.random.default_rng(seed)
        hist = []
        for e in range(epochs):
            order = rng.permutation(len(graphs))
            losses = [self.train_step(graphs[i], lr * lr_decay ** e) for i in order]
            hist.append(float(np.mean(losses)))
        return hist


def training_targets(results: list[SolveResult]) -> list[WarmStart]:
    return [WarmStart.from_result(r) for r in results]


@dataclass
class WarmSolveInfo:
    warm_iterations: list[int]
    choices: list[str]          # per LP: "network", "hint", "blend" or "cold" (the certified start)
    start_kkt: list[float]      # the chosen start's relative KKT error
    fallbacks: int
    predict_s: float
    certify_s: float
    solve_s: float
    fallback_s: float
    probe_iterations: int = 0   # iterations spent on the probes, all candidates counted


def probe_candidates(models: list[ModelIR], sets: list[list], options: PdhgOptions, iterations: int):
    """Runs `iterations` PDHG iterations from every candidate start of every LP
    (one batch of all of them) and returns the points reached, per candidate
    set, with None kept for candidates that do not exist."""
    o = dataclasses.replace(options, tolerance=0.0, max_iterations=iterations,
                            check_frequency=min(options.check_frequency, iterations))
    flat, where = [], []
    for p, st in enumerate(sets):
        for i, w in enumerate(st):
            if w is not None or p == len(sets) - 1:   # the last set (cold) is always probed
                flat.append(i)
                where.append((p, i, w))
    res = solve_batch([models[i] for i in flat], o, warm=[w for _, _, w in where])
    out = [[None] * len(models) for _ in sets]
    for (p, i, _), r in zip(where, res):
        out[p][i] = WarmStart(r.x, r.y, 0.0)
    return out, len(flat) * iterations


def select_starts(models: list[ModelIR], candidates: dict[str, list], device: int = 0,
                  probe_iterations: int = 0, options: PdhgOptions | None = None):
    """The certificate decides: for every LP, the candidate start with the
    smallest FP64 relative KKT error (max of primal, dual and gap) among
    ``candidates`` (name -> one point or None per LP), with the cold start
    always among them.  With ``probe_iterations`` > 0 every candidate is first
    advanced that many PDHG iterations (``options``) and judged, and returned,
    at the point it reached: a start whose error is small but whose
    neighbourhood converges slowly loses to one that moves faster.  Returns
    (starts, names, kkt, probe iterations spent)."""
    from .certificate import certify_batch

    names = list(candidates) + ["cold"]
    sets = [candidates[nm] for nm in candidates] + [[None] * len(models)]
    spent = 0
    if probe_iterations > 0:
        if options is None:
            raise ValueError("select_starts: probing needs the solver options")
        sets, spent = probe_candidates(models, sets, options, probe_iterations)
    certs = certify_batch(models, sets, device)
    starts, chosen, kkt = [], [], []
    for i in range(len(models)):
        best = len(names) - 1
        for p in range(len(names) - 1):
            if sets[p][i] is not None and certs[p][i].kkt < certs[best][i].kkt:
                best = p
        starts.append(sets[best][i])
        chosen.append(names[best])
        kkt.append(certs[best][i].kkt)
    return starts, chosen, kkt, spent


def splice_refinement(hint: WarmStart | None, pred: WarmStart | None, mask) -> WarmStart | None:
    """The hint with the network's values where ``mask`` = (x_mask, y_mask) is
    set (None: the network's point everywhere)."""
    if hint is None or pred is None or mask is None:
        return pred
    xm, ym = mask
    x = np.where(xm, pred.x, np.asarray(hint.x, np.float64))
    y = None if hint.y is None else np.where(ym, pred.y, np.asarray(hint.y, np.float64))
    return WarmStart(x, y, 0.0)


def warm_solve_batch(models: list[ModelIR], net: WarmStartNet, options: PdhgOptions,
                     fallback_iterations: int | None = None,
                     hints: list[WarmStart | None] | None = None,
                     use_predicted_weight: bool = False,
                     probe_iterations: int = 0,
                     refine_masks: list | None = None,
                     select: bool = True) -> tuple[list[SolveResult], WarmSolveInfo]:
    """Learned warm start, certified, with the cold start as fallback.

    1. The network predicts (x, y, omega) for every LP (refining ``hints``
       when given, see ``GnnGraph``).  With ``refine_masks`` (one
       (x_mask, y_mask) or None per LP) its point is taken only where the
       mask is set and the hint elsewhere (``splice_refinement``): on
       rolling-horizon windows the network then predicts the tail of the
       horizon, which the previous window's solution cannot supply, and
       leaves the periods that solution already has to it.
    2. With ``select`` the certificate decides the start of each LP: the
       network's point, the hint, (when probing) the point halfway between
       them, or the cold start, whichever has the smallest FP64 relative KKT
       error (``select_starts``), judged after ``probe_iterations`` PDHG
       iterations from each when that is > 0 (the solve then continues from
       the chosen probe's point; every probe's iterations are counted in
       ``WarmSolveInfo.probe_iterations``).  Without ``select`` every LP
       starts from the network's point (the cold start where there is none).
    3. The batch is solved from those starts (with the predicted primal
       weight when ``use_predicted_weight``, else the solver's default).
    4. Every LP whose solve is not optimal (it hit ``options.max_iterations``)
       is solved again from the cold start with ``fallback_iterations``
       (default: the same limit).
    Every answer is judged by the same relative-KKT criterion as a cold solve."""
    import time

    t0 = time.perf_counter()
    pred = net.predict(models, hints=hints)
    if refine_masks is not None:
        if hints is None or len(refine_masks) != len(models):
            raise ValueError("warm_solve_batch: refine_masks needs hints and one mask (or None) per LP")
        pred = [splice_refinement(h, p, mk) for h, p, mk in zip(hints, pred, refine_masks)]
    t1 = time.perf_counter()
    cands = {"network": pred}
    if not select:
        res, info = _solve_from(models, options, pred, ["network" if p is not None else "cold" for p in pred],
                                [float("nan")] * len(models), pred, use_predicted_weight, fallback_iterations,
                                t0, t1, time.perf_counter(), 0)
        return res, info
    if hints is not None:
        cands["hint"] = list(hints)
        # halfway between the hint and the network's refinement of it: the
        # network's corrections are right on average, and often too large
        if probe_iterations > 0:
            cands["blend"] = [None if (h is None or p is None) else
                              WarmStart(0.5 * (np.asarray(h.x) + p.x), 0.5 * (np.asarray(h.y) + p.y), 0.0)
                              for h, p in zip(hints, pred)]
    starts, chosen, kkt, spent = select_starts(models, cands, net.device, probe_iterations, options)
    return _solve_from(models, options, starts, chosen, kkt, pred, use_predicted_weight, fallback_iterations,
                       t0, t1, time.perf_counter(), spent)


def _solve_from(models, options, starts, chosen, kkt, pred, use_predicted_weight, fallback_iterations,
                t0, t1, t_sel, spent):
    """Steps 3 and 4 of ``warm_solve_batch``."""
    import time

    warm = []
    for st, p in zip(starts, pred):
        if st is None:
            warm.append(None)
        else:
            w = p.primal_weight if (use_predicted_weight and p is not None) else 0.0
            warm.append(WarmStart(st.x, st.y, w))
    t2 = t_sel
    res = solve_batch(models, options, warm=warm)
    t3 = time.perf_counter()
    warm_its = [r.iterations for r in res]
    bad = [i for i, r in enumerate(res) if r.status != SolveStatus.kOptimal and models[i].numVars() > 0]
    if bad:
        o = dataclasses.replace(options)
        if fallback_iterations:
            o.max_iterations = fallback_iterations
        cold = solve_batch([models[i] for i in bad], o)
        for i, r in zip(bad, cold):
            if r.status == SolveStatus.kOptimal or res[i].status != SolveStatus.kOptimal:
                res[i] = r
    t4 = time.perf_counter()
    return res, WarmSolveInfo(warm_its, chosen, kkt, len(bad), t1 - t0, t2 - t1, t3 - t2, t4 - t3, spent)
