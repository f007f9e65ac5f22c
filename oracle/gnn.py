"""NumPy restatement of the warm-start network (test infrastructure only).

The network has no counterpart in the reference; this module is the checker
the GPU forward and backward passes are compared against.  It restates the
definition in pramaan_b200/csrc/gnn.cuh: graph scales and node features,
three message-passing layers of width 64, the x / y / primal-weight heads,
the loss, and its gradient with respect to every parameter.

Two arithmetic modes:
  * ``exact=True``  — float64 throughout, no rounding: the gradient is the
    true derivative of the loss, which the CPU tests pin against central
    finite differences;
  * ``exact=False`` — float32 with BF16 rounding at the points the GPU rounds
    (parameters, every activation h and aggregation, the dense-layer input
    gradients dz), the mode the GPU tests compare with.
Parity is "unpinned" against any reference: the reference has no learned
component.  Only tests/ may import this module.
"""
from __future__ import annotations

import numpy as np

H = 64
FEAT = 9
LAYERS = 3
LOSS_FLOOR = 1e-2

# flat parameter layout (gnn.cuh GnnParams)
VIN_W = 0
VIN_B = VIN_W + 64 * FEAT
CIN_W = VIN_B + 64
CIN_B = CIN_W + 64 * FEAT
LAYER0 = CIN_B + 64
DENSE_W = 64 * 128
LAYER_STRIDE = 2 * (DENSE_W + 64)
HEAD_X = LAYER0 + LAYERS * LAYER_STRIDE
HEAD_Y = HEAD_X + 65
HEAD_W = HEAD_Y + 65
COUNT = HEAD_W + 129


def layer_w(l: int, side: int) -> int:
    return LAYER0 + l * LAYER_STRIDE + side * (DENSE_W + 64)


def layer_b(l: int, side: int) -> int:
    return layer_w(l, side) + DENSE_W


def bf16(a) -> np.ndarray:
    """Round float32 values to the nearest BF16 (ties to even), as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


class Graph:
    """Packed batch of LPs (LPs without variables are skipped), as GnnGraph."""

    def __init__(self, models, targets=None, hints=None):
        self.index = [k for k, md in enumerate(models) if md.numVars() > 0]
        ms = [models[k] for k in self.index]
        self.K = len(ms)
        self.r0 = np.cumsum([0] + [md.numRows() for md in ms])
        self.c0 = np.cumsum([0] + [md.numVars() for md in ms])
        self.m, self.n = int(self.r0[-1]), int(self.c0[-1])
        rows, cols, vals = [], [], []
        cost, vlo, vhi, rlo, rhi = [], [], [], [], []
        self.s_a, self.s_b, self.s_c, self.omega_ref = (np.ones(self.K) for _ in range(4))
        for q, md in enumerate(ms):
            sign = -1.0 if int(md.obj_sense) == 1 else 1.0
            cnt = np.diff(md.row_ptr)
            rows.append(np.repeat(np.arange(md.numRows()), cnt) + self.r0[q])
            cols.append(md.col_idx.astype(np.int64) + self.c0[q])
            vals.append(md.values)
            c = sign * md.obj_coeffs
            cost.append(c)
            vlo.append(md.var_lower)
            vhi.append(md.var_upper)
            rlo.append(md.row_lower)
            rhi.append(md.row_upper)
            lo, hi = md.row_lower, md.row_upper
            fl, fu = lo > -1e29, hi < 1e29
            bvals = np.concatenate([lo[fl], hi[fu & ~(fl & (lo == hi))]])
            sa = np.sqrt(np.mean(md.values ** 2)) if md.nnz() else 0.0
            sb = np.sqrt(np.mean(bvals ** 2)) if len(bvals) else 0.0
            sc = np.sqrt(np.mean(c ** 2))
            self.s_a[q] = sa if sa > 0 and np.isfinite(sa) else 1.0
            self.s_b[q] = sb if sb > 0 and np.isfinite(sb) else 1.0
            self.s_c[q] = sc if sc > 0 and np.isfinite(sc) else 1.0
            cn, bn = np.sqrt(np.sum(c ** 2)), np.sqrt(np.sum(bvals ** 2))
            self.omega_ref[q] = cn / bn if cn > 1e-10 and bn > 1e-10 and np.isfinite(cn / bn) else 1.0
        cat = lambda v, dt: np.concatenate(v).astype(dt) if v else np.zeros(0, dt)  # noqa: E731
        self.rows, self.cols, self.vals = cat(rows, np.int64), cat(cols, np.int64), cat(vals, np.float64)
        self.cost, self.vlo, self.vhi = cat(cost, np.float64), cat(vlo, np.float64), cat(vhi, np.float64)
        self.rlo, self.rhi = cat(rlo, np.float64), cat(rhi, np.float64)
        self.lp_col = np.repeat(np.arange(self.K), np.diff(self.c0))
        self.lp_row = np.repeat(np.arange(self.K), np.diff(self.r0))
        self.deg_r = np.bincount(self.rows, minlength=self.m)
        self.deg_c = np.bincount(self.cols, minlength=self.n)
        sa_e = self.s_a[self.lp_row[self.rows]] if len(self.rows) else np.zeros(0)
        self.coef_r = self.vals / (sa_e * np.maximum(1, self.deg_r[self.rows]))
        self.coef_c = self.vals / (sa_e * np.maximum(1, self.deg_c[self.cols]))
        self.base_x, self.base_y = np.zeros(self.n), np.zeros(self.m)
        self.hint_x, self.hint_y = np.zeros(self.n, bool), np.zeros(self.m, bool)
        if hints is not None:
            for q, k in enumerate(self.index):
                h = hints[k]
                if h is None:
                    continue
                sa, sb, sc = self.s_a[q], self.s_b[q], self.s_c[q]
                if h.x is not None:
                    self.base_x[self.c0[q]:self.c0[q + 1]] = np.asarray(h.x) * sa / sb
                    self.hint_x[self.c0[q]:self.c0[q + 1]] = True
                if h.y is not None and self.r0[q + 1] > self.r0[q]:
                    self.base_y[self.r0[q]:self.r0[q + 1]] = np.asarray(h.y) * sa / sc
                    self.hint_y[self.r0[q]:self.r0[q + 1]] = True
        # the device adds the hint terms in FP32
        self.base_x = self.base_x.astype(np.float32).astype(np.float64)
        self.base_y = self.base_y.astype(np.float32).astype(np.float64)
        self.fv, self.fc = self._features()
        self.has_targets = targets is not None
        if targets is not None:
            tx, ty, tw = np.zeros(self.n), np.zeros(self.m), np.zeros(self.K)
            for q, k in enumerate(self.index):
                t = targets[k]
                sa, sb, sc = self.s_a[q], self.s_b[q], self.s_c[q]
                tx[self.c0[q]:self.c0[q + 1]] = np.asarray(t.x) * sa / sb
                if self.r0[q + 1] > self.r0[q]:
                    ty[self.r0[q]:self.r0[q + 1]] = np.asarray(t.y) * sa / sc
                tw[q] = np.log(t.primal_weight / self.omega_ref[q])
            self.tx, self.ty, self.tw = tx, ty, tw
            # per-LP loss weights (float32 on the device)
            nk, mk = np.diff(self.c0), np.diff(self.r0)
            tx32, ty32 = tx.astype(np.float32).astype(np.float64), ty.astype(np.float32).astype(np.float64)
            sx = np.bincount(self.lp_col, weights=tx32 ** 2, minlength=self.K)
            sy = np.bincount(self.lp_row, weights=ty32 ** 2, minlength=self.K)
            self.lw_x = (1.0 / (nk * (sx / nk + LOSS_FLOOR))).astype(np.float32).astype(np.float64)
            self.lw_y = np.where(mk > 0, 1.0 / (np.maximum(mk, 1) * (sy / np.maximum(mk, 1) + LOSS_FLOOR)), 0.0)
            self.lw_y = self.lw_y.astype(np.float32).astype(np.float64)

    def _features(self):
        clip = lambda v: np.clip(v, -10.0, 10.0)  # noqa: E731
        sa_c, sb_c, sc_c = self.s_a[self.lp_col], self.s_b[self.lp_col], self.s_c[self.lp_col]
        absum_c = np.bincount(self.cols, weights=np.abs(self.vals), minlength=self.n)
        fl, fu = self.vlo > -1e29, self.vhi < 1e29
        fv = np.zeros((self.n, FEAT))
        fv[:, 0] = self.cost / sc_c
        fv[:, 1], fv[:, 2] = fl, fu
        fv[:, 3] = np.where(fl, clip(np.where(fl, self.vlo, 0) * sa_c / sb_c), 0)
        fv[:, 4] = np.where(fu, clip(np.where(fu, self.vhi, 0) * sa_c / sb_c), 0)
        fv[:, 5] = np.log1p(self.deg_c) / 4.0
        fv[:, 6] = np.where(self.deg_c > 0, absum_c / (sa_c * np.maximum(self.deg_c, 1)), 0)
        fv[:, 7] = self.hint_x
        fv[:, 8] = clip(self.base_x)
        sa_r, sb_r = self.s_a[self.lp_row], self.s_b[self.lp_row]
        absum_r = np.bincount(self.rows, weights=np.abs(self.vals), minlength=self.m)
        fl, fu = self.rlo > -1e29, self.rhi < 1e29
        fc = np.zeros((self.m, FEAT))
        fc[:, 0] = fl & fu & (self.rlo == self.rhi)
        fc[:, 1], fc[:, 2] = fl, fu
        fc[:, 3] = np.where(fl, clip(np.where(fl, self.rlo, 0) / sb_r), 0)
        fc[:, 4] = np.where(fu, clip(np.where(fu, self.rhi, 0) / sb_r), 0)
        fc[:, 5] = np.log1p(self.deg_r) / 4.0
        fc[:, 6] = np.where(self.deg_r > 0, absum_r / (sa_r * np.maximum(self.deg_r, 1)), 0)
        fc[:, 7] = self.hint_y
        fc[:, 8] = clip(self.base_y)
        return fv.astype(np.float32), fc.astype(np.float32)


class _Arith:
    def __init__(self, exact: bool):
        self.exact = exact
        self.dt = np.float64 if exact else np.float32

    def r(self, a):
        return np.asarray(a, self.dt) if self.exact else bf16(a)

    def a(self, a):
        return np.asarray(a, self.dt)


def _agg(rows, cols, coef, src, out_rows, ar):
    """out[r] = sum_e coef[e] src[cols[e]] over entries e with rows[e] == r."""
    out = np.zeros((out_rows, src.shape[1]), ar.dt)
    if len(rows):
        np.add.at(out, rows, (coef.astype(ar.dt)[:, None] * src[cols]).astype(ar.dt))
    return out


def forward(params, g: Graph, exact: bool = False) -> dict:
    """Activations of the network on graph g (dict of arrays, packed order)."""
    ar = _Arith(exact)
    p = ar.r(np.asarray(params, np.float32) if not exact else np.asarray(params, np.float64))
    fv, fc = ar.a(g.fv), ar.a(g.fc)
    wv, bv = p[VIN_W:VIN_B].reshape(64, FEAT), p[VIN_B:VIN_B + 64]
    wc, bc = p[CIN_W:CIN_B].reshape(64, FEAT), p[CIN_B:CIN_B + 64]
    hv = ar.r(np.maximum(fv @ wv.T + bv, 0))
    hc = ar.r(np.maximum(fc @ wc.T + bc, 0))
    act = {"hv0": hv, "hc0": hc, "xc": [], "xv": []}
    for l in range(LAYERS):
        agg_c = ar.r(_agg(g.rows, g.cols, g.coef_r, hv, g.m, ar))
        xc = np.concatenate([hc, agg_c], axis=1)
        W, b = p[layer_w(l, 0):layer_b(l, 0)].reshape(64, 128), p[layer_b(l, 0):layer_b(l, 0) + 64]
        hc = ar.r(np.maximum(xc @ W.T + b, 0))
        agg_v = ar.r(_agg(g.cols, g.rows, g.coef_c, hc, g.n, ar))
        xv = np.concatenate([hv, agg_v], axis=1)
        W, b = p[layer_w(l, 1):layer_b(l, 1)].reshape(64, 128), p[layer_b(l, 1):layer_b(l, 1) + 64]
        hv = ar.r(np.maximum(xv @ W.T + b, 0))
        act["xc"].append(xc)
        act["xv"].append(xv)
    act["hc3"], act["hv3"] = hc, hv
    act["xhat"] = ar.a(g.base_x) + (hv @ p[HEAD_X:HEAD_X + 64] + p[HEAD_X + 64])
    act["yhat"] = ar.a(g.base_y) + (hc @ p[HEAD_Y:HEAD_Y + 64] + p[HEAD_Y + 64])
    pooled = np.zeros((g.K, 128), ar.dt)
    for q in range(g.K):
        pooled[q, :64] = hv[g.c0[q]:g.c0[q + 1]].sum(0) / (g.c0[q + 1] - g.c0[q])
        if g.r0[q + 1] > g.r0[q]:
            pooled[q, 64:] = hc[g.r0[q]:g.r0[q + 1]].sum(0) / (g.r0[q + 1] - g.r0[q])
    act["pooled"] = pooled
    act["rho"] = pooled @ p[HEAD_W:HEAD_W + 128] + p[HEAD_W + 128]
    act["p"] = p
    return act


def loss_and_grad(params, g: Graph, exact: bool = False, grad: bool = True):
    """(loss, gradient) of the definition in gnn.cuh on graph g."""
    ar = _Arith(exact)
    a = forward(params, g, exact)
    p = a["p"]
    K = g.K
    inv_n = 1.0 / np.diff(g.c0)
    inv_m = np.where(np.diff(g.r0) > 0, 1.0 / np.maximum(np.diff(g.r0), 1), 0.0)
    ex = a["xhat"] - g.tx
    ey = a["yhat"] - g.ty
    ew = a["rho"] - g.tw
    lx = np.bincount(g.lp_col, weights=ex ** 2, minlength=K) * g.lw_x
    ly = np.bincount(g.lp_row, weights=ey ** 2, minlength=K) * g.lw_y
    loss = float(np.sum(lx + ly + ew ** 2) / K)
    if not grad:
        return loss, None
    G = np.zeros(COUNT, np.float64)
    dx = ar.a(2 * ex * g.lw_x[g.lp_col] / K)
    dy = ar.a(2 * ey * g.lw_y[g.lp_row] / K)
    drho = ar.a(2 * ew / K)
    hv, hc = a["hv3"], a["hc3"]
    G[HEAD_X:HEAD_X + 64] = dx @ hv
    G[HEAD_X + 64] = dx.sum()
    G[HEAD_Y:HEAD_Y + 64] = dy @ hc
    G[HEAD_Y + 64] = dy.sum()
    G[HEAD_W:HEAD_W + 128] = drho @ a["pooled"]
    G[HEAD_W + 128] = drho.sum()
    wx, wy, ww = p[HEAD_X:HEAD_X + 64], p[HEAD_Y:HEAD_Y + 64], p[HEAD_W:HEAD_W + 128]
    dhv = ar.a(dx[:, None] * wx[None, :] + (drho * inv_n)[g.lp_col][:, None] * ww[None, :64])
    dhc = ar.a(dy[:, None] * wy[None, :] + (drho * inv_m)[g.lp_row][:, None] * ww[None, 64:])
    outs_c = [a["xc"][l + 1][:, :64] if l + 1 < LAYERS else a["hc3"] for l in range(LAYERS)]
    outs_v = [a["xv"][l + 1][:, :64] if l + 1 < LAYERS else a["hv3"] for l in range(LAYERS)]
    for l in reversed(range(LAYERS)):
        # variable side
        dz = ar.r(np.where(outs_v[l] > 0, dhv, 0))
        G[layer_b(l, 1):layer_b(l, 1) + 64] = dz.sum(0)
        G[layer_w(l, 1):layer_b(l, 1)] = (dz.T @ a["xv"][l]).ravel()
        W = p[layer_w(l, 1):layer_b(l, 1)].reshape(64, 128)
        dX = ar.a(dz @ W)
        dhv, dagg = dX[:, :64].copy(), dX[:, 64:]
        # agg_v backward: dh_c[i] += sum_j coef_c(i, j) dagg_v[j]
        dhc = dhc + _agg(g.rows, g.cols, g.coef_c, dagg, g.m, ar)
        # constraint side
        dz = ar.r(np.where(outs_c[l] > 0, dhc, 0))
        G[layer_b(l, 0):layer_b(l, 0) + 64] = dz.sum(0)
        G[layer_w(l, 0):layer_b(l, 0)] = (dz.T @ a["xc"][l]).ravel()
        W = p[layer_w(l, 0):layer_b(l, 0)].reshape(64, 128)
        dX = ar.a(dz @ W)
        dhc, dagg = dX[:, :64].copy(), dX[:, 64:]
        # agg_c backward: dh_v[j] += sum_i coef_r(i, j) dagg_c[i]
        dhv = dhv + _agg(g.cols, g.rows, g.coef_r, dagg, g.n, ar)
    dz0 = np.where(a["hv0"] > 0, dhv, 0)
    G[VIN_W:VIN_B] = (dz0.T @ ar.a(g.fv)).ravel()
    G[VIN_B:VIN_B + 64] = dz0.sum(0)
    dz0 = np.where(a["hc0"] > 0, dhc, 0)
    G[CIN_W:CIN_B] = (dz0.T @ ar.a(g.fc)).ravel()
    G[CIN_B:CIN_B + 64] = dz0.sum(0)
    return loss, G


def init_params(seed: int = 0) -> np.ndarray:
    """He-uniform weights, zero biases, small random heads: a NumPy
    initialisation for tests (the library's own starts its heads at zero)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(COUNT)
    p[VIN_W:VIN_B] = rng.uniform(-1, 1, 64 * FEAT) * np.sqrt(6 / FEAT)
    p[CIN_W:CIN_B] = rng.uniform(-1, 1, 64 * FEAT) * np.sqrt(6 / FEAT)
    for l in range(LAYERS):
        for side in range(2):
            p[layer_w(l, side):layer_b(l, side)] = rng.uniform(-1, 1, DENSE_W) * np.sqrt(6 / 128)
    p[HEAD_X:HEAD_X + 64] = rng.uniform(-0.1, 0.1, 64)
    p[HEAD_Y:HEAD_Y + 64] = rng.uniform(-0.1, 0.1, 64)
    p[HEAD_W:HEAD_W + 128] = rng.uniform(-0.1, 0.1, 128)
    return p   # (non-zero heads, so that every gradient block is exercised)


def trace_layout(g: Graph) -> list[tuple[str, tuple]]:
    """Names and shapes of pramaan_gnn_forward_trace's output, in order."""
    out = [(f"xc{l}", (g.m, 128)) for l in range(LAYERS)]
    out += [(f"xv{l}", (g.n, 128)) for l in range(LAYERS)]
    out += [("hc3", (g.m, 64)), ("hv3", (g.n, 64)), ("xhat", (g.n,)), ("yhat", (g.m,)),
            ("pooled", (g.K, 128)), ("rho", (g.K,))]
    return out
