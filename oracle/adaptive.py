"""CPU restatement (numpy/scipy, FP64) of the library's adaptive restarted
PDHG — TEST INFRASTRUCTURE ONLY.

Mirrors pramaan_b200/csrc/pdhg_adaptive.cu step for step so the GPU mode can
be checked on small LPs: Ruiz (10 simultaneous row/column inf-norm passes) +
Pock-Chambolle (alpha = 1) steps folded into per-element steps, eta = 0.99 /
||Sigma^1/2 A T^1/2|| by power iteration, primal weight omega (initially
||C c|| / ||R b||), the reference's dual-first update with those steps,
uniform averages since the last restart, and KKT-based restarts
(0.2 / 0.8 / 0.36) with the omega update exp(0.5 log(dy/dx) + 0.5 log omega).
The algorithm is PDLP's (Applegate et al., NeurIPS 2021) as restated in the
library; the relative KKT is oracle/pdhg_oracle.c orc_rel_kkt in numpy.

This restatement runs in FP64 on the untranslated iterates.  The library
runs the same iteration on FP32 corrections around FP64 master iterates that
absorb the correction at every restart; in exact arithmetic that translation
changes nothing, so this is the method the device code approximates, and
the device results are compared with it through the properties that survive
FP32 rounding (step size, initial primal weight, relative KKT at the answer).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

INF = 1e29


def _csr(model):
    return sp.csr_matrix((model.values, model.col_idx, model.row_ptr),
                         shape=(model.numRows(), model.numVars()))


def problem(model):
    sgn = -1.0 if int(model.obj_sense) == 1 else 1.0
    A = _csr(model)
    return dict(A=A, AT=A.T.tocsr(), c=sgn * model.obj_coeffs, rl=model.row_lower, ru=model.row_upper,
                vl=model.var_lower, vu=model.var_upper)


def rel_kkt(P, x, y):
    """Relative KKT pieces (pr2, dr2, pobj, dobj, rel_p, rel_d, rel_gap)."""
    A, c, rl, ru, vl, vu = P["A"], P["c"], P["rl"], P["ru"], P["vl"], P["vu"]
    act = A @ x
    d = np.where((rl > -INF) & (act < rl), rl - act, 0.0) + np.where((ru < INF) & (act > ru), act - ru, 0.0)
    pr2 = float(d @ d)
    dvar = np.where((vl > -INF) & (x < vl), vl - x, 0.0) + np.where((vu < INF) & (x > vu), x - vu, 0.0)
    pr2 += float(dvar @ dvar)
    lam = -y
    dobj = float(np.sum(np.where((lam > 0) & (rl > -INF), lam * rl, 0.0)) +
                 np.sum(np.where((lam < 0) & (ru < INF), lam * ru, 0.0)))
    dr2 = float(np.sum(np.where((lam > 0) & ~(rl > -INF), lam * lam, 0.0)) +
                np.sum(np.where((lam < 0) & ~(ru < INF), lam * lam, 0.0)))
    rc = c + P["AT"] @ y
    dobj += float(np.sum(np.where((rc > 0) & (vl > -INF), rc * vl, 0.0)) +
                  np.sum(np.where((rc < 0) & (vu < INF), rc * vu, 0.0)))
    dr2 += float(np.sum(np.where((rc > 0) & ~(vl > -INF), rc * rc, 0.0)) +
                 np.sum(np.where((rc < 0) & ~(vu < INF), rc * rc, 0.0)))
    pobj = float(c @ x)
    b2 = float(np.sum(np.where(rl > -INF, rl * rl, 0.0)) +
               np.sum(np.where((ru < INF) & ~((rl > -INF) & (rl == ru)), ru * ru, 0.0)))
    return dict(pr2=pr2, dr2=dr2, pobj=pobj, dobj=dobj,
                rel_p=np.sqrt(pr2) / (1 + np.sqrt(b2)), rel_d=np.sqrt(dr2) / (1 + np.linalg.norm(c)),
                rel_gap=abs(pobj - dobj) / (1 + abs(pobj) + abs(dobj)))


def weighted(k, omega):
    gap = k["pobj"] - k["dobj"]
    return np.sqrt(omega * omega * k["pr2"] + k["dr2"] / (omega * omega) + gap * gap)


def steps(P, passes=10):
    """Ruiz scales (R, C) and the Pock-Chambolle steps mapped to the original variables."""
    A = P["A"]
    m, n = A.shape
    R, C = np.ones(m), np.ones(n)
    absA = abs(A).tocsr()
    for _ in range(passes):
        S = sp.diags(R) @ absA @ sp.diags(C)
        rmax = np.asarray(S.max(axis=1).todense()).ravel() if m else np.zeros(0)
        cmax = np.asarray(S.max(axis=0).todense()).ravel() if n else np.zeros(0)
        R = np.where(rmax > 0, R / np.sqrt(np.maximum(rmax, 1e-300)), R)
        C = np.where(cmax > 0, C / np.sqrt(np.maximum(cmax, 1e-300)), C)
    S = sp.diags(R) @ absA @ sp.diags(C)
    rs = np.asarray(S.sum(axis=1)).ravel()
    cs = np.asarray(S.sum(axis=0)).ravel()
    sigma = np.where(rs > 1e-30, R * R / np.maximum(rs, 1e-300), R * R)
    tau = np.where(cs > 1e-30, C * C / np.maximum(cs, 1e-300), C * C)
    return R, C, sigma, tau


def op_norm(P, sigma, tau, iters=40):
    A, AT = P["A"], P["AT"]
    n = A.shape[1]
    v = np.full(n, 1.0 / np.sqrt(n))
    st = np.sqrt(tau)
    lam = 0.0
    for it in range(iters):
        w = st * (AT @ (sigma * (A @ (st * v))))
        prev, lam = lam, float(v @ w)
        wn = np.linalg.norm(w)
        if not wn > 0:
            break
        v = w / wn
        if it > 5 and abs(lam - prev) <= 1e-4 * abs(lam):
            break
    return np.sqrt(lam) if lam > 0 else 1.0


def initial_weight(P, R, C):
    """omega_0 = ||C c|| / ||R b|| on the Ruiz-scaled problem (1 when either is ~0)."""
    c, rl, ru = P["c"], P["rl"], P["ru"]
    cs = np.linalg.norm(c * C)
    bvec = np.concatenate([np.where(rl > -INF, rl * R, 0.0),
                           np.where((ru < INF) & ~((rl > -INF) & (rl == ru)), ru * R, 0.0)])
    bs = np.linalg.norm(bvec)
    return cs / bs if cs > 1e-10 and bs > 1e-10 else 1.0


def solve(model, tol=1e-6, max_iterations=100000, check_frequency=64, return_trace=False):
    P = problem(model)
    A, AT, c = P["A"], P["AT"], P["c"]
    m, n = A.shape
    R, C, sigma, tau = steps(P)
    eta = 0.99 / op_norm(P, sigma, tau)
    rl, ru, vl, vu = P["rl"], P["ru"], P["vl"], P["vu"]
    omega = initial_weight(P, R, C)
    x = np.clip(0.0, vl, vu) * np.ones(n)
    xbar = x.copy()
    y = np.zeros(m)
    xs, ys, cnt = np.zeros(n), np.zeros(m), 0
    xl, yl = x.copy(), y.copy()
    k = rel_kkt(P, x, y)
    kkt_restart, kkt_prev = weighted(k, omega), np.inf
    last_restart, it, restarts = 0, 0, 0
    trace = []
    status = "iteration_limit"
    while it < max_iterations:
        for _ in range(min(check_frequency, max_iterations - it)):
            s = sigma * eta * omega
            w = y / s + A @ xbar
            y = s * (w - np.clip(w, rl, ru))
            t = tau * eta / omega
            xn = np.clip(x - t * (c + AT @ y), vl, vu)
            xbar = 2 * xn - x
            x = xn
            xs += x
            ys += y
            cnt += 1
            it += 1
        xa, ya = xs / cnt, ys / cnt
        kc, ka = rel_kkt(P, x, y), rel_kkt(P, xa, ya)
        trace.append((it, kc["rel_p"], kc["rel_d"], kc["rel_gap"], omega))
        if kc["rel_p"] <= tol and kc["rel_d"] <= tol and kc["rel_gap"] <= tol:
            status = "optimal"
            break
        if ka["rel_p"] <= tol and ka["rel_d"] <= tol and ka["rel_gap"] <= tol:
            x, y, status = xa, ya, "optimal"
            break
        wc, wa = weighted(kc, omega), weighted(ka, omega)
        use_avg = wa < wc
        kcand = min(wa, wc)
        restart = (kcand <= 0.2 * kkt_restart or (kcand <= 0.8 * kkt_restart and kcand > kkt_prev)
                   or (it - last_restart) >= 0.36 * it)
        kkt_prev = kcand
        if restart:
            if use_avg:
                x, y = xa.copy(), ya.copy()
            xbar = x.copy()
            xs[:], ys[:], cnt = 0.0, 0.0, 0
            dx = np.linalg.norm((x - xl) / C)
            dy = np.linalg.norm((y - yl) / R) if m else 0.0
            if dx > 1e-10 and dy > 1e-10:
                omega = float(np.exp(0.5 * np.log(dy / dx) + 0.5 * np.log(omega)))
            xl, yl = x.copy(), y.copy()
            kkt_restart, kkt_prev, last_restart = kcand, np.inf, it
            restarts += 1
    out = dict(status=status, iterations=it, x=x, y=y, restarts=restarts, omega=omega, eta=eta,
               kkt=rel_kkt(P, x, y))
    if return_trace:
        out["trace"] = trace
    return out


def solve_halpern(model, tol=1e-6, max_iterations=100000, check_frequency=64, rho=1.0):
    """The library's PRAMAAN_ALGO_HALPERN mode restated in FP64.

    Same preconditioned steps, step size and initial primal weight as
    ``solve``; the PDHG operator taken primal first,
        x+ = clip(x - t (c + A^T y)),  y+ = dual step of y with A (2 x+ - x),
    each iteration moving to w ((1 + rho) T(z) - rho z) + (1 - w) z_anchor with
    w = (k + 1) / (k + 2), k the iterations since the last restart (restarted
    Halpern PDHG with reflection, Lu and Yang 2024).  At every check
    (``check_frequency`` iterations) the fixed-point residual
    r = sqrt(sum (dx)^2 / t + sum (dy)^2 / s) of the interval's first and last
    iteration is known; an LP restarts at its current iterate when r_last <=
    0.2 r0, or r_last <= 0.8 r0 and r_last grew since the previous check, or
    0.36 of all iterations passed since its last restart (r0: the residual
    of the first iteration after the restart); the primal weight is updated
    at restarts as in ``solve``; termination on the relative KKT of the
    current iterate."""
    P = problem(model)
    A, AT, c = P["A"], P["AT"], P["c"]
    m, n = A.shape
    R, C, sigma, tau = steps(P)
    eta = 0.99 / op_norm(P, sigma, tau)
    rl, ru, vl, vu = P["rl"], P["ru"], P["vl"], P["vu"]
    omega = initial_weight(P, R, C)
    x = np.clip(0.0, vl, vu) * np.ones(n)
    y = np.zeros(m)
    xa, ya = x.copy(), y.copy()
    k = rel_kkt(P, x, y)
    it, restarts, last_restart, kk = 0, 0, 0, 0
    r0, rprev, need_r0 = 0.0, np.inf, True
    status = "iteration_limit"
    if k["rel_p"] <= tol and k["rel_d"] <= tol and k["rel_gap"] <= tol:
        status = "optimal"
    while status != "optimal" and it < max_iterations:
        s, t = sigma * eta * omega, tau * eta / omega
        chunk = min(check_frequency, max_iterations - it)
        r_first = r_last = 0.0
        for j in range(chunk):
            xt = np.clip(x - t * (c + AT @ y), vl, vu)
            w_ = y / s + A @ (2 * xt - x)
            yt = s * (w_ - np.clip(w_, rl, ru))
            r = np.sqrt(np.sum((x - xt) ** 2 / t) + np.sum((y - yt) ** 2 / s))
            if j == 0:
                r_first = r
            if j == chunk - 1:
                r_last = r
            wgt = (kk + 1) / (kk + 2)
            x = wgt * ((1 + rho) * xt - rho * x) + (1 - wgt) * xa
            y = wgt * ((1 + rho) * yt - rho * y) + (1 - wgt) * ya
            kk += 1
            it += 1
        if need_r0:
            r0, need_r0 = r_first, False
        k = rel_kkt(P, x, y)
        if k["rel_p"] <= tol and k["rel_d"] <= tol and k["rel_gap"] <= tol:
            status = "optimal"
            break
        restart = (r_last <= 0.2 * r0 or (r_last <= 0.8 * r0 and r_last > rprev)
                   or (it - last_restart) >= 0.36 * it)
        rprev = r_last
        if restart:
            dx = np.linalg.norm((x - xa) / C)
            dy = np.linalg.norm((y - ya) / R) if m else 0.0
            if dx > 1e-10 and dy > 1e-10:
                omega = float(np.exp(0.5 * np.log(dy / dx) + 0.5 * np.log(omega)))
            xa, ya = x.copy(), y.copy()
            kk, last_restart, restarts = 0, it, restarts + 1
            rprev, need_r0 = np.inf, True
    return dict(status=status, iterations=it, x=x, y=y, restarts=restarts, omega=omega, eta=eta,
                kkt=rel_kkt(P, x, y))
