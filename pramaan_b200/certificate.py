"""FP64 certificates of LP solutions computed on the GPU (pramaan_certify_batch).

The first three fields restate the reference certificate
(pramaan::generate_certificate, src/certificate/certificate.cpp:23-107):
objective, maximum row violation and maximum variable-bound violation.  The
rest add the dual side the reference leaves empty: the FP64 relative KKT error
of the point (x, y) — the quantity that decides whether a warm start or a
solution is accepted.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .pdhg import ModelIR, _f64, _ptr


@dataclass
class Certificate:
    objective_value: float
    primal_residual: float
    bound_violation: float
    rel_primal: float
    rel_dual: float
    rel_gap: float
    primal_objective: float
    dual_objective: float
    kkt: float


def certify_batch(models: list[ModelIR], points: list[list], device: int = 0) -> list[list[Certificate]]:
    """Certificates of every point set: ``points[p][k]`` is point p of LP k, an
    object with ``x`` and ``y`` (arrays or None; x None is the solver's cold
    start clamp(0, l, u), y None is 0) or None for the cold start itself.
    Returns ``out[p][k]``."""
    k = len(models)
    P = len(points)
    if k == 0 or P == 0:
        return [[] for _ in range(P)]
    lps = (L.CLp * k)()
    for i, md in enumerate(models):
        lps[i] = md.c_struct()
    arr = (L.CWarmStart * (k * P))()
    keep = []
    for p, row in enumerate(points):
        if len(row) != k:
            raise ValueError("every point set needs one entry per model")
        for i, w in enumerate(row):
            x = None if w is None or getattr(w, "x", None) is None else _f64(w.x)
            y = None if w is None or getattr(w, "y", None) is None else _f64(w.y)
            if x is not None and len(x) != models[i].numVars():
                raise ValueError("point x has the wrong length")
            if y is not None and len(y) != models[i].numRows():
                raise ValueError("point y has the wrong length")
            keep.extend([x, y])
            arr[p * k + i].x, arr[p * k + i].y, arr[p * k + i].primal_weight = _ptr(x), _ptr(y), 0.0
    out = (L.CCertificate * (k * P))()
    L.check(L.lib().pramaan_certify_batch(lps, k, arr, P, device, out))
    res = []
    for p in range(P):
        res.append([Certificate(*[getattr(out[p * k + i], f) for f, _ in L.CCertificate._fields_])
                    for i in range(k)])
    return res


def certify(model: ModelIR, x, y=None, device: int = 0) -> Certificate:
    """Certificate of one point of one LP."""
    class _P:
        pass
    pt = _P()
    pt.x, pt.y = np.asarray(x, np.float64), None if y is None else np.asarray(y, np.float64)
    return certify_batch([model], [[pt]], device)[0][0]
