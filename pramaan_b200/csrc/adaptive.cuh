// adaptive.cuh — epilogues and reductions of the adaptive restarted PDHG
// (PRAMAAN_ALGO_ADAPTIVE).
//
// The adaptive mode keeps the reference's per-element diagonal iteration
// (the same dual/primal update formulas) and adds, after PDLP (Applegate et
// al., NeurIPS 2021) and cuPDLP.jl (Lu & Yang, 2023):
//   * Ruiz + Pock-Chambolle preconditioning, folded into the per-element
//     steps (sigma_i = R_i^2 sigma'_i, tau_j = C_j^2 tau'_j), so the matrix is
//     never rewritten;
//   * a step size eta from a power-iteration estimate of the preconditioned
//     operator norm and a primal weight omega, applied through two device
//     scalars (eta*omega on the dual side, eta/omega on the primal side) so
//     a captured graph stays valid when omega changes;
//   * running FP64 sums of the iterates (the averaged iterate);
//   * relative-KKT evaluation of the current and averaged iterates in FP64,
//     with deterministic per-block partial sums.
#pragma once

#include "epilogues.cuh"

namespace pb {

// Partial-sum layout: one row of kPartSlots doubles per block; rows
// [0, kPartMain) belong to the main SpMV kernel (channel 0), rows
// [kPartMain, kPartMain + kPartFix) to its fixup kernel (channel 1).
constexpr int kPartMain = 1024;
constexpr int kPartFix = 2048;
constexpr int kPartRows = kPartMain + kPartFix;
constexpr int kPartSlots = 16;

template <int K>
__device__ __forceinline__ void block_sums_to(const double (&v)[K], double* __restrict__ part, int channel,
                                              int slot0) {
    __shared__ double s_part[32][K];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double w[K];
#pragma unroll
    for (int k = 0; k < K; ++k) w[k] = warp_sum(v[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) s_part[warp][k] = w[k];
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            double t = lane < nw ? s_part[lane][k] : 0.0;
            t = warp_sum(t);
            if (lane == 0) part[size_t(channel * kPartMain + blockIdx.x) * kPartSlots + slot0 + k] = t;
        }
    }
    __syncthreads();
}

// The adaptive iteration runs on corrections around FP64 master iterates
// (x = x_m + d, y = y_m + e; pdhg_adaptive.cu folds d, e into the master at
// every restart).  Everything the update needs from the master is folded
// into FP32 vectors when the master changes:
//   r_lo = A x_m - l_r,  r_hi = A x_m - u_r   (+-1e30 where the bound is infinite)
//   c'   = c + A^T y_m,  l'_x = l_x - x_m,  u'_x = u_x - x_m.
//
// Dual update (the reference's, src/gpu/pdhg_kernels.cuh:72-89, with the
// adaptive step s = sigma_i * scal[1]) in a form that keeps FP32 precision
// when y/s is much larger than A x̄:
//   w = y/s + (A x̄)_i  only decides the case;
//   w > u_r:  y' = y + s ((A x̄)_i - u_r)    w < l_r:  y' = y + s ((A x̄)_i - l_r)
//   else:     y' = 0
// which is s (w - clamp(w, l_r, u_r)) rearranged.  In correction form
// (A x̄ = A x_m + A d̄, y = y_m + e) the residual differences come straight
// from r_lo / r_hi and the inactive case is e' = -y_m.  Adds e' to the
// running FP64 sum of the epoch's average.
struct EpiDualAdapt {
    const float* __restrict__ sigma;
    const float* __restrict__ r_lo;
    const float* __restrict__ r_hi;
    const float* __restrict__ y_m;   // FP32 copy of the master dual
    float* __restrict__ e;
    double* __restrict__ esum;
    const float* __restrict__ scal;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int i) const {
        prefetch_l2(sigma + i); prefetch_l2(r_lo + i); prefetch_l2(r_hi + i); prefetch_l2(y_m + i);
        prefetch_l2(e + i); prefetch_l2(esum + i);
    }
    __device__ void apply(State&, int i, float ad) const {
        const float s = __fmul_rn(sigma[i], scal[1]);
        float en = e[i];
        if (s > 0.0f) {
            const float ym = y_m[i];
            const float q = __fdiv_rn(__fadd_rn(ym, en), s);
            const float hi = __fadd_rn(ad, r_hi[i]);   // (A x̄)_i - u_r
            const float lo = __fadd_rn(ad, r_lo[i]);   // (A x̄)_i - l_r
            if (__fadd_rn(q, hi) > 0.0f) en = __fmaf_rn(s, hi, en);
            else if (__fadd_rn(q, lo) < 0.0f) en = __fmaf_rn(s, lo, en);
            else en = -ym;
        }
        e[i] = en;
        esum[i] += static_cast<double>(en);
    }
    __device__ void finish(State&, int) const {}
};

// Primal update of the reference (src/gpu/pdhg_kernels.cuh:95-109) with the
// adaptive step tau_j * scal[0], plus the running sum of x.  On corrections
// the same formula applies to d with c' and the shifted bounds l'_x, u'_x.
struct EpiPrimalAdapt {
    const float* __restrict__ tau;
    const float* __restrict__ c;
    const float* __restrict__ l_x;
    const float* __restrict__ u_x;
    float* __restrict__ x;
    float* __restrict__ x_bar;
    double* __restrict__ xsum;
    const float* __restrict__ scal;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int j) const {
        prefetch_l2(tau + j); prefetch_l2(c + j); prefetch_l2(l_x + j); prefetch_l2(u_x + j);
        prefetch_l2(x + j); prefetch_l2(xsum + j);
    }
    __device__ void apply(State&, int j, float aty) const {
        const float x_prev = x[j];
        const float g = __fadd_rn(c[j], aty);
        const float step = __fmaf_rn(-__fmul_rn(tau[j], scal[0]), g, x_prev);
        const float x_new = fminf(fmaxf(step, l_x[j]), u_x[j]);
        x_bar[j] = __fmaf_rn(2.0f, x_new, -x_prev);
        x[j] = x_new;
        xsum[j] += static_cast<double>(x_new);
    }
    __device__ void finish(State&, int) const {}
};

// ---- restarted Halpern PDHG with reflection -------------------------------
// The PDHG operator T is taken primal first,
//   x+ = clip(x - tau (c + A^T y), l_x, u_x),   y+ = dual step of y with A (2 x+ - x),
// and each iteration moves to the Halpern point with reflection rho = 1:
//   z <- w ((1 + rho) T(z) - rho z) + (1 - w) z_anchor,   w = (k + 1) / (k + 2),
// k = iterations since the LP's last restart (Lu and Yang, "Restarted Halpern
// PDHG for linear programming", 2024).  On FP32 corrections around FP64
// master iterates the anchor (the restart point) is the master itself, so the
// anchor term vanishes (anchor == nullptr).  The fixed-point residual
// ||z - T(z)||^2 in the step-weighted norm (sum (dx)^2/tau + (dy)^2/sigma) is
// written per element on the iterations that ask for it (fpr != nullptr).
constexpr float kHalpernReflection = 1.0f;

// Halpern weight of LP q at iteration offset of the interval.
__device__ __forceinline__ float halpern_weight_lp(const int* iter_base, int offset, const int* restart_iter, int q) {
    const long long k = (long long)(*iter_base) + offset - restart_iter[q];
    return k <= 0 ? 0.5f : float(double(k + 1) / double(k + 2));
}
__device__ __forceinline__ float halpern_weight(const int* iter_base, int offset, const int* restart_iter,
                                                const int* lp, int i) {
    return halpern_weight_lp(iter_base, offset, restart_iter, lp ? lp[i] : 0);   // lp null: one LP
}

struct EpiPrimalHalpern {
    const float* __restrict__ tau;
    const float* __restrict__ c;
    const float* __restrict__ l_x;
    const float* __restrict__ u_x;
    float* __restrict__ x;
    float* __restrict__ x_bar;
    const float* __restrict__ anchor;      // nullptr: 0
    const int* __restrict__ lp;
    const int* __restrict__ restart_iter;
    const int* __restrict__ iter_base;
    int offset;
    double* __restrict__ fpr;              // nullptr: not this iteration
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int j) const {
        prefetch_l2(tau + j); prefetch_l2(c + j); prefetch_l2(l_x + j); prefetch_l2(u_x + j);
        prefetch_l2(x + j); if (lp) prefetch_l2(lp + j);
    }
    // apply() split in two: every input of column j, then the update
    // (the tile loop loads several columns ahead of their updates).
    static constexpr bool kSplit = true;
    struct In { float x_prev, t, c, lo, hi, a, w; };
    // w: the Halpern weight of column j's LP (halpern_weight), when the
    // caller has it already
    __device__ In load(int j, float w) const {
        In in;
        in.x_prev = x[j];
        in.t = tau[j];
        in.c = c[j];
        in.lo = l_x[j];
        in.hi = u_x[j];
        in.a = anchor ? anchor[j] : 0.0f;
        in.w = w;
        return in;
    }
    __device__ In load(int j) const { return load(j, halpern_weight(iter_base, offset, restart_iter, lp, j)); }
    __device__ void store(State&, int j, const In& in, float aty) const {
        if (!(in.t > 0.0f)) {        // a frozen LP keeps its iterate
            x_bar[j] = in.x_prev;
            if (fpr) fpr[j] = 0.0;
            return;
        }
        const float g = __fadd_rn(in.c, aty);
        const float xt = fminf(fmaxf(__fmaf_rn(-in.t, g, in.x_prev), in.lo), in.hi);
        x_bar[j] = __fmaf_rn(2.0f, xt, -in.x_prev);
        const float refl = __fmaf_rn(1.0f + kHalpernReflection, xt, -kHalpernReflection * in.x_prev);
        x[j] = __fmaf_rn(in.w, __fsub_rn(refl, in.a), in.a);
        if (fpr) {
            const double d = double(in.x_prev) - double(xt);
            fpr[j] = d * d / double(in.t);
        }
    }
    __device__ void apply(State& st, int j, float aty) const { store(st, j, load(j), aty); }
    __device__ void finish(State&, int) const {}
};

struct EpiDualHalpern {
    const float* __restrict__ sigma;
    const float* __restrict__ r_lo;
    const float* __restrict__ r_hi;
    const float* __restrict__ y_m;         // FP32 copy of the master dual
    float* __restrict__ e;
    const float* __restrict__ anchor;      // nullptr: 0
    const int* __restrict__ lp;
    const int* __restrict__ restart_iter;
    const int* __restrict__ iter_base;
    int offset;
    double* __restrict__ fpr;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int i) const {
        prefetch_l2(sigma + i); prefetch_l2(r_lo + i); prefetch_l2(r_hi + i); prefetch_l2(y_m + i);
        prefetch_l2(e + i); if (lp) prefetch_l2(lp + i);
    }
    static constexpr bool kSplit = true;
    struct In { float s, e_prev, ym, hi, lo, a, w; };
    __device__ In load(int i, float w) const {
        In in;
        in.s = sigma[i];
        in.e_prev = e[i];
        in.ym = y_m[i];
        in.hi = r_hi[i];
        in.lo = r_lo[i];
        in.a = anchor ? anchor[i] : 0.0f;
        in.w = w;
        return in;
    }
    __device__ In load(int i) const { return load(i, halpern_weight(iter_base, offset, restart_iter, lp, i)); }
    __device__ void store(State&, int i, const In& in, float ad) const {
        const float s = in.s;
        const float e_prev = in.e_prev;
        float en = e_prev;
        if (s > 0.0f) {
            const float ym = in.ym;
            const float q = __fdiv_rn(__fadd_rn(ym, e_prev), s);
            const float hi = __fadd_rn(ad, in.hi);
            const float lo = __fadd_rn(ad, in.lo);
            if (__fadd_rn(q, hi) > 0.0f) en = __fmaf_rn(s, hi, e_prev);
            else if (__fadd_rn(q, lo) < 0.0f) en = __fmaf_rn(s, lo, e_prev);
            else en = -ym;
        }
        const float refl = __fmaf_rn(1.0f + kHalpernReflection, en, -kHalpernReflection * e_prev);
        e[i] = __fmaf_rn(in.w, __fsub_rn(refl, in.a), in.a);
        if (fpr) {
            const double d = double(e_prev) - double(en);
            fpr[i] = s > 0.0f ? d * d / double(s) : 0.0;
        }
    }
    __device__ void apply(State& st, int i, float ad) const { store(st, i, load(i), ad); }
    __device__ void finish(State&, int) const {}
};

// Row part of the relative KKT error (FP64, on the original problem in
// minimisation form; lambda = -y since y is the reference's negated
// multiplier) of x = x_m + d, y = y_m + e: the SpMV delivers (A d)_i, the
// master's activity A x_m is added in FP64.  Sums the squared distance of
// (A x)_i to [row_lower, row_upper], the dual objective's row terms, and the
// squared dual infeasibility of a multiplier sign that pairs with an
// infinite row bound.
struct EpiRowKkt {
    const double* __restrict__ row_lo;
    const double* __restrict__ row_hi;
    const double* __restrict__ act_m;   // A x_m
    const double* __restrict__ y_m;
    const float* __restrict__ e;
    double* __restrict__ part;
    int slot0;
    struct State { double pr2, dr2, dobj, bad; };
    __device__ void init(State& s) const { s.pr2 = s.dr2 = s.dobj = s.bad = 0.0; }
    __device__ void prefetch(int i) const {
        prefetch_l2(row_lo + i); prefetch_l2(row_hi + i); prefetch_l2(act_m + i); prefetch_l2(y_m + i);
        prefetch_l2(e + i);
    }
    __device__ void apply(State& s, int i, double ad) const {
        const double lo = row_lo[i], hi = row_hi[i];
        const double act = act_m[i] + ad;
        if (!isfinite(act)) { s.bad = 1.0; return; }
        const bool lo_f = lo > -1e29, hi_f = hi < 1e29;
        double d = 0.0;
        if (lo_f && act < lo) d = lo - act;
        if (hi_f && act > hi) d = act - hi;
        s.pr2 += d * d;
        const double lam = -(y_m[i] + static_cast<double>(e[i]));
        if (lam > 0.0) { if (lo_f) s.dobj += lam * lo; else s.dr2 += lam * lam; }
        else if (lam < 0.0) { if (hi_f) s.dobj += lam * hi; else s.dr2 += lam * lam; }
    }
    __device__ void finish(State& s, int channel) const {
        const double v[4] = {s.pr2, s.dr2, s.dobj, s.bad};
        block_sums_to<4>(v, part, channel, slot0);
    }
};

// Column part: reduced cost rc = c + A^T y = rc_m + (A^T e)_j with the
// master's rc_m = c + A^T y_m in FP64, the dual objective's bound terms, the
// squared dual infeasibility of an rc sign that pairs with an infinite
// variable bound, the primal objective c^T x, and x's bound violation
// (x = x_m + d; FP32 rounding can leave it just outside an FP64 bound).
struct EpiColKkt {
    const double* __restrict__ c;
    const double* __restrict__ var_lo;
    const double* __restrict__ var_hi;
    const double* __restrict__ rc_m;
    const double* __restrict__ x_m;
    const float* __restrict__ d;
    double* __restrict__ part;
    int slot0;
    struct State { double pr2, dr2, dobj, pobj; };
    __device__ void init(State& s) const { s.pr2 = s.dr2 = s.dobj = s.pobj = 0.0; }
    __device__ void prefetch(int j) const {
        prefetch_l2(c + j); prefetch_l2(var_lo + j); prefetch_l2(var_hi + j); prefetch_l2(rc_m + j);
        prefetch_l2(x_m + j); prefetch_l2(d + j);
    }
    __device__ void apply(State& s, int j, double ate) const {
        const double lo = var_lo[j], hi = var_hi[j], cj = c[j];
        const double xj = x_m[j] + static_cast<double>(d[j]);
        const bool lo_f = lo > -1e29, hi_f = hi < 1e29;
        const double rc = rc_m[j] + ate;
        if (rc > 0.0) { if (lo_f) s.dobj += rc * lo; else s.dr2 += rc * rc; }
        else if (rc < 0.0) { if (hi_f) s.dobj += rc * hi; else s.dr2 += rc * rc; }
        s.pobj += cj * xj;
        double v = 0.0;
        if (lo_f && xj < lo) v = lo - xj;
        if (hi_f && xj > hi) v = xj - hi;
        s.pr2 += v * v;
    }
    __device__ void finish(State& s, int channel) const {
        const double v[4] = {s.pr2, s.dr2, s.dobj, s.pobj};
        block_sums_to<4>(v, part, channel, slot0);
    }
};

// y[r] = scale[r] * value (power iteration).
struct EpiStoreScaled {
    float* __restrict__ y;
    const float* __restrict__ scale;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int) const {}
    __device__ void apply(State&, int r, float v) const { y[r] = scale[r] * v; }
    __device__ void finish(State&, int) const {}
};

}  // namespace pb
