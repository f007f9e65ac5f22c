"""Seeded synthetic LP generators with the shapes of the benchmark configs.

All generators build feasible LPs by construction (x0 feasible, and
(y0, s0 >= 0) dual feasible):  min c^T x  s.t.  A x = b,  0 <= x <= u  with
x0 ~ U(0,1), b = A x0, y0 ~ N(0,1), s0 ~ U(0,1), c = A^T y0 + s0,
u = x0 + U(1,5).  Matrix values are FP32-representable numbers stored as
FP64 (the ModelIR value type).

* ``random_sparse_lp``  — "4 non-zeros per column at uniform random rows,
  values N(0,1)" (the 1000 x 3000 plain-PDHG workload; any size).
* ``zipf_lp``           — power-law rows: lengths Zipf(s) capped, uniform
  distinct columns, values N(0,1) times log-uniform row scales (the
  2,000,000 x 5,000,000 SpMV-roofline workload; any size).  Runs in torch on
  any device so the large instance is generated on the GPU in about a second.
* ``ill_conditioned_lp`` — k non-zeros per column with log-uniform row and
  column scales (the 200,000 x 500,000 precision-ladder workload).
* ``rolling_horizon_lp`` / ``rolling_horizon_batch`` — production planning
  over T periods and P products (the batched workload: 512 LPs with
  T ~ U{24..336}, P ~ U{5..50}).
"""
from __future__ import annotations

import numpy as np

from .pdhg import ModelIR, ObjSense


def _csr_from_coo(rows: np.ndarray, cols: np.ndarray, vals: np.ndarray, m: int):
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    counts = np.bincount(rows, minlength=m)
    row_ptr = np.zeros(m + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return row_ptr.astype(np.int32), cols.astype(np.int32), vals


def _distinct_rows_per_col(rng: np.random.Generator, m: int, n: int, k: int) -> np.ndarray:
    """(n, k) array of row indices, distinct within each column."""
    k = min(k, m)
    r = rng.integers(0, m, size=(n, k))
    while True:
        s = np.sort(r, axis=1)
        dup_cols = np.nonzero((s[:, 1:] == s[:, :-1]).any(axis=1))[0]
        if dup_cols.size == 0:
            return r
        r[dup_cols] = rng.integers(0, m, size=(dup_cols.size, k))


def _feasible_model(rng, m, n, row_ptr, col_idx, vals) -> tuple[ModelIR, dict]:
    rows = np.repeat(np.arange(m), np.diff(row_ptr))
    x0 = rng.random(n)
    b = np.bincount(rows, weights=vals * x0[col_idx], minlength=m)
    y0 = rng.standard_normal(m)
    s0 = rng.random(n)
    c = np.bincount(col_idx, weights=vals * y0[rows], minlength=n) + s0
    u = x0 + rng.uniform(1.0, 5.0, size=n)
    model = ModelIR(c, row_ptr, col_idx, vals, b, b.copy(), np.zeros(n), u, ObjSense.kMinimize, 0.0)
    return model, dict(x0=x0, y0=y0, s0=s0)


def random_sparse_lp(m: int = 1000, n: int = 3000, nnz_per_col: int = 4, seed: int = 0,
                     return_certificate: bool = False):
    """Equality-constrained random sparse LP with k non-zeros per column."""
    rng = np.random.default_rng(seed)
    r = _distinct_rows_per_col(rng, m, n, nnz_per_col)
    cols = np.repeat(np.arange(n), r.shape[1])
    rows = r.reshape(-1)
    vals = rng.standard_normal(rows.size).astype(np.float32).astype(np.float64)
    row_ptr, col_idx, vals = _csr_from_coo(rows, cols, vals, m)
    model, cert = _feasible_model(rng, m, n, row_ptr, col_idx, vals)
    return (model, cert) if return_certificate else model


def ill_conditioned_lp(m: int = 200_000, n: int = 500_000, nnz_per_col: int = 8, seed: int = 0,
                       scale_exp: float = 4.0, return_certificate: bool = False):
    """Random sparse LP with row and column scales log-uniform in
    [10^-scale_exp, 10^scale_exp] (condition ~ 10^(4 scale_exp))."""
    rng = np.random.default_rng(seed)
    r = _distinct_rows_per_col(rng, m, n, nnz_per_col)
    cols = np.repeat(np.arange(n), r.shape[1])
    rows = r.reshape(-1)
    rs = 10.0 ** rng.uniform(-scale_exp, scale_exp, size=m)
    cs = 10.0 ** rng.uniform(-scale_exp, scale_exp, size=n)
    vals = (rng.standard_normal(rows.size) * rs[rows] * cs[cols]).astype(np.float32).astype(np.float64)
    row_ptr, col_idx, vals = _csr_from_coo(rows, cols, vals, m)
    model, cert = _feasible_model(rng, m, n, row_ptr, col_idx, vals)
    return (model, cert) if return_certificate else model


def zipf_lp(m: int = 2_000_000, n: int = 5_000_000, s: float = 1.5, cap: int = 5000,
            seed: int = 0, scale_lo: float = 1e-2, scale_hi: float = 1e2, device: str = "cpu",
            as_tensors: bool = False):
    """Power-law-row LP (torch on `device`).

    Row lengths ~ Zipf(s) truncated to [1, cap]; columns uniform, distinct
    within a row (duplicates drawn by chance are merged away, so the actual
    nnz is reported by the result); values FP32(N(0,1) * row scale) with row
    scales log-uniform in [scale_lo, scale_hi].  Returns a ModelIR (host) or,
    with as_tensors=True, a dict of torch tensors on `device`.
    """
    import torch

    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    cap = min(cap, n)
    k = torch.arange(1, cap + 1, dtype=torch.float64, device=dev)
    cdf = torch.cumsum(k.pow(-s), 0)
    cdf = cdf / cdf[-1]
    u = torch.rand(m, generator=g, dtype=torch.float64, device=dev)
    lens = (torch.searchsorted(cdf, u) + 1).clamp_(1, cap)
    rows = torch.repeat_interleave(torch.arange(m, device=dev), lens)
    cols = torch.randint(0, n, (rows.numel(),), generator=g, device=dev)
    key = rows * n + cols
    del rows, cols
    key, _ = torch.sort(key)
    keep = torch.ones_like(key, dtype=torch.bool)
    keep[1:] = key[1:] != key[:-1]
    key = key[keep]
    del keep
    rows = torch.div(key, n, rounding_mode="floor")
    cols = (key - rows * n).to(torch.int32)
    del key
    nnz = cols.numel()
    counts = torch.bincount(rows, minlength=m)
    row_ptr = torch.zeros(m + 1, dtype=torch.int64, device=dev)
    torch.cumsum(counts, 0, out=row_ptr[1:])
    return _lp_on_structure(rows, cols, row_ptr, m, n, g, dev, scale_lo, scale_hi, as_tensors)


def _lp_on_structure(rows, cols, row_ptr, m, n, g, dev, scale_lo, scale_hi, as_tensors):
    """Values, a feasible point and bounded costs on a given structure (torch
    tensors: rows int64 and cols int32 per entry in CSR order, row_ptr int64).
    Values FP32(N(0,1) * row scale), row scales log-uniform in
    [scale_lo, scale_hi]; b = A x0 with x0 ~ U(0,1) in [0, ub]; c = A^T y0 + s0
    with s0 > 0, so the LP is feasible and bounded."""
    import torch

    nnz = cols.numel()
    lo, hi = np.log10(scale_lo), np.log10(scale_hi)
    rscale = torch.pow(10.0, lo + (hi - lo) * torch.rand(m, generator=g, dtype=torch.float64, device=dev))
    vals = (torch.randn(nnz, generator=g, dtype=torch.float64, device=dev) * rscale[rows]).float().double()
    x0 = torch.rand(n, generator=g, dtype=torch.float64, device=dev)
    b = torch.zeros(m, dtype=torch.float64, device=dev).index_add_(0, rows, vals * x0[cols.long()])
    y0 = torch.randn(m, generator=g, dtype=torch.float64, device=dev)
    s0 = torch.rand(n, generator=g, dtype=torch.float64, device=dev)
    c = torch.zeros(n, dtype=torch.float64, device=dev).index_add_(0, cols.long(), vals * y0[rows]) + s0
    del rows
    ub = x0 + 1.0 + 4.0 * torch.rand(n, generator=g, dtype=torch.float64, device=dev)
    t = dict(row_ptr=row_ptr.to(torch.int32), col_idx=cols, values=vals, obj_coeffs=c,
             row_lower=b, row_upper=b.clone(), var_lower=torch.zeros(n, dtype=torch.float64, device=dev),
             var_upper=ub, x0=x0, y0=y0, s0=s0)
    if as_tensors:
        return t
    h = {k2: v.cpu().numpy() for k2, v in t.items()}
    return ModelIR(h["obj_coeffs"], h["row_ptr"], h["col_idx"], h["values"], h["row_lower"],
                   h["row_upper"], h["var_lower"], h["var_upper"], ObjSense.kMinimize, 0.0)


def banded_lp(m: int = 2_000_000, n: int = 5_000_000, per_row: int = 54, band: int = 256, seed: int = 0,
              scale_lo: float = 1e-2, scale_hi: float = 1e2, device: str = "cpu", as_tensors: bool = False):
    """LP whose rows couple nearby columns (torch on `device`).

    Row i draws `per_row` columns uniformly within +-band of i*n/m (clamped to
    [0, n); duplicates merged, so the actual nnz is reported by the result):
    the locally coupled structure of multi-period and network models ordered
    by period or node.  Values, bounds and costs as zipf_lp.  Returns a
    ModelIR (host) or, with as_tensors=True, a dict of torch tensors.
    """
    import torch

    dev = torch.device(device)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    rows = torch.arange(m, device=dev).repeat_interleave(per_row)
    center = torch.div(rows * n, m, rounding_mode="floor")
    cols = (center + torch.randint(-band, band + 1, (rows.numel(),), generator=g, device=dev)).clamp_(0, n - 1)
    del center
    key = rows * n + cols
    del rows, cols
    key, _ = torch.sort(key)
    keep = torch.ones_like(key, dtype=torch.bool)
    keep[1:] = key[1:] != key[:-1]
    key = key[keep]
    del keep
    rows = torch.div(key, n, rounding_mode="floor")
    cols = (key - rows * n).to(torch.int32)
    del key
    counts = torch.bincount(rows, minlength=m)
    row_ptr = torch.zeros(m + 1, dtype=torch.int64, device=dev)
    torch.cumsum(counts, 0, out=row_ptr[1:])
    return _lp_on_structure(rows, cols, row_ptr, m, n, g, dev, scale_lo, scale_hi, as_tensors)


def model_from_tensors(t: dict) -> ModelIR:
    h = {k: v.cpu().numpy() for k, v in t.items() if k in (
        "obj_coeffs", "row_ptr", "col_idx", "values", "row_lower", "row_upper", "var_lower", "var_upper")}
    return ModelIR(h["obj_coeffs"], h["row_ptr"], h["col_idx"], h["values"], h["row_lower"],
                   h["row_upper"], h["var_lower"], h["var_upper"], ObjSense.kMinimize, 0.0)


def rolling_horizon_lp(T: int, P: int, seed: int = 0, demand=None, rng=None, cost=None, cap=None):
    """Multi-product production planning over T periods.

    Variables per (product p, period t), in three blocks of P*T (index
    p*T + t inside a block): produce x >= 0, inventory I >= 0, backlog B >= 0.
    Rows: inventory balance per (p, t) (row p*T + t, an equality)
        I[p,t-1] - B[p,t-1] + x[p,t] - I[p,t] + B[p,t] = d[p,t]
    (no t-1 terms at t = 0) and one shared capacity row per period
    (row P*T + t):  sum_p x[p,t] <= cap[t].
    Demand d ~ lognormal(mu=3, sigma=0.5) unless given as a (P, T) array;
    production, holding and backlog costs ~ U(1, 10) per (p, t) unless given
    (3 blocks of P*T, index p*T + t); cap[t] = U(0.8, 1.2) * sum_p E[d]
    unless given.  Backlog keeps every instance
    feasible and positive costs keep it bounded.
    """
    rng = rng if rng is not None else np.random.default_rng(seed)
    PT = P * T
    if demand is None:
        demand = rng.lognormal(3.0, 0.5, size=(P, T))
    demand = np.asarray(demand, np.float64).reshape(P, T)
    if cost is None:
        cost = rng.uniform(1.0, 10.0, size=3 * PT)
    cost = np.asarray(cost, np.float64).reshape(3 * PT)
    mean_d = np.exp(3.0 + 0.125)
    if cap is None:
        cap = rng.uniform(0.8, 1.2, size=T) * P * mean_d
    cap = np.asarray(cap, np.float64).reshape(T)
    p_idx, t_idx = np.divmod(np.arange(PT), T)
    # balance rows: columns x, I[t-1], I[t], B[t-1], B[t] (ascending)
    first = t_idx == 0
    cnt = np.where(first, 3, 5)
    row_ptr = np.zeros(PT + T + 1, np.int64)
    row_ptr[1:PT + 1] = np.cumsum(cnt)
    cols = np.empty(int(row_ptr[PT]), np.int64)
    vals = np.empty(int(row_ptr[PT]), np.float64)
    base = row_ptr[:PT]
    q = np.arange(PT)
    # first period: x, I, B
    f = q[first]
    cols[base[f]], vals[base[f]] = f, 1.0
    cols[base[f] + 1], vals[base[f] + 1] = PT + f, -1.0
    cols[base[f] + 2], vals[base[f] + 2] = 2 * PT + f, 1.0
    g = q[~first]
    cols[base[g]], vals[base[g]] = g, 1.0
    cols[base[g] + 1], vals[base[g] + 1] = PT + g - 1, 1.0
    cols[base[g] + 2], vals[base[g] + 2] = PT + g, -1.0
    cols[base[g] + 3], vals[base[g] + 3] = 2 * PT + g - 1, -1.0
    cols[base[g] + 4], vals[base[g] + 4] = 2 * PT + g, 1.0
    # capacity rows: x[p, t] for p = 0..P-1
    cap_cols = (np.arange(P)[None, :] * T + np.arange(T)[:, None]).ravel()
    row_ptr[PT + 1:] = row_ptr[PT] + P * np.arange(1, T + 1)
    cols = np.concatenate([cols, cap_cols])
    vals = np.concatenate([vals, np.ones(P * T)])
    m, n = PT + T, 3 * PT
    inf = 1e30
    row_lower = np.concatenate([demand.ravel(), np.full(T, -inf)])
    row_upper = np.concatenate([demand.ravel(), cap])
    return ModelIR(cost, row_ptr.astype(np.int32), cols.astype(np.int32), vals, row_lower, row_upper,
                   np.zeros(n), np.full(n, inf), ObjSense.kMinimize, 0.0)


def rolling_horizon_batch(count: int = 512, seed: int = 0, T_range=(24, 336), P_range=(5, 50)):
    """``count`` rolling-horizon LPs with T ~ U{T_range}, P ~ U{P_range}
    (inclusive), drawn from one seeded stream."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        T = int(rng.integers(T_range[0], T_range[1] + 1))
        P = int(rng.integers(P_range[0], P_range[1] + 1))
        out.append(rolling_horizon_lp(T, P, rng=rng))
    return out


def rolling_horizon_stream(count: int, seed: int = 0, T: int | None = None, P: int | None = None,
                           T_range=(24, 336), P_range=(5, 50), phi: float = 0.9, sigma: float = 0.1):
    """``count`` consecutive windows of one production-planning stream.

    Window k is ``rolling_horizon_lp`` over periods k .. k+T-1 of one long
    horizon (the window shifts by one period from LP to LP).  T and P are
    drawn from the batch ranges unless given.  Demand of product p in period
    t is mu_p exp(u_{p,t}) with mu_p ~ lognormal(3, 0.5) and u an AR(1)
    process, u_t = phi u_{t-1} + sigma e_t (stationary start); production,
    holding and backlog costs ~ U(1, 10) and the capacity
    U(0.8, 1.2) * sum_p E[d] are drawn per period of the long horizon, so
    consecutive windows share all but one period of their data."""
    rng = np.random.default_rng(seed)
    T = int(rng.integers(T_range[0], T_range[1] + 1)) if T is None else int(T)
    P = int(rng.integers(P_range[0], P_range[1] + 1)) if P is None else int(P)
    L = T + count - 1
    mu = rng.lognormal(3.0, 0.5, size=P)
    u = np.empty((P, L))
    u[:, 0] = rng.normal(0.0, sigma / np.sqrt(1.0 - phi * phi), size=P)
    eps = rng.normal(0.0, sigma, size=(P, L))
    for t in range(1, L):
        u[:, t] = phi * u[:, t - 1] + eps[:, t]
    demand = mu[:, None] * np.exp(u)
    cost = rng.uniform(1.0, 10.0, size=(3, P, L))
    cap = rng.uniform(0.8, 1.2, size=L) * P * np.exp(3.0 + 0.125)
    out = []
    for k in range(count):
        sl = slice(k, k + T)
        out.append(rolling_horizon_lp(T, P, demand=demand[:, sl], cost=cost[:, :, sl].reshape(-1),
                                      cap=cap[sl]))
    return out


def rolling_horizon_shift(x, y, T: int, P: int):
    """A window's solution mapped onto the next window of its stream.

    In the layout of ``rolling_horizon_lp`` (variables in three blocks of
    P*T with index p*T + t; balance rows p*T + t, then T capacity rows) the
    next window covers periods 1..T of this one: every period moves one slot
    earlier and the new last period repeats the old last one.  Returns
    (x', y') as float64 arrays (y' is None when y is None)."""
    def sh(a, lead):
        a = np.asarray(a, np.float64).reshape(*lead, T)
        return np.concatenate([a[..., 1:], a[..., -1:]], axis=-1).ravel()

    xs = sh(x, (3, P))
    if y is None:
        return xs, None
    y = np.asarray(y, np.float64)
    ys = np.concatenate([sh(y[:P * T], (P,)), sh(y[P * T:], (1,))])
    return xs, ys


def rolling_horizon_tail_mask(T: int, P: int, k: int):
    """(x_mask, y_mask) of the last k periods of a window in the layout of
    ``rolling_horizon_lp``: the periods a shifted previous solution knows
    least about (the new last period is only a copy, and the ones before it
    carried the previous window's end-of-horizon effects)."""
    k = max(0, min(int(k), T))
    tail = np.zeros(T, bool)
    tail[T - k:] = True
    return np.tile(tail, 3 * P), np.concatenate([np.tile(tail, P), tail])
