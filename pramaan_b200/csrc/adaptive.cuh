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

// Dual update of the reference (src/gpu/pdhg_kernels.cuh:72-89) with the
// adaptive step sigma_i * scal[1], plus the running sum of y.
struct EpiDualAdapt {
    const float* __restrict__ sigma;
    const float* __restrict__ l_r;
    const float* __restrict__ u_r;
    float* __restrict__ y;
    double* __restrict__ ysum;
    const float* __restrict__ scal;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int i) const {
        prefetch_l2(sigma + i); prefetch_l2(l_r + i); prefetch_l2(u_r + i); prefetch_l2(y + i);
        prefetch_l2(ysum + i);
    }
    __device__ void apply(State&, int i, float ax) const {
        const float sig = __fmul_rn(sigma[i], scal[1]);
        float yn = y[i];
        if (sig > 0.0f) {
            const float w = __fadd_rn(__fdiv_rn(yn, sig), ax);
            const float wp = fminf(fmaxf(w, l_r[i]), u_r[i]);
            yn = __fmul_rn(sig, __fsub_rn(w, wp));
        }
        y[i] = yn;
        ysum[i] += static_cast<double>(yn);
    }
    __device__ void finish(State&, int) const {}
};

// Primal update of the reference (src/gpu/pdhg_kernels.cuh:95-109) with the
// adaptive step tau_j * scal[0], plus the running sum of x.
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

// Row part of the relative KKT error (FP64, on the original problem in
// minimisation form; lambda = -y since y is the reference's negated
// multiplier): squared distance of (A x)_i to [row_lower, row_upper], the
// dual objective's row terms, and the squared dual infeasibility of a
// multiplier sign that pairs with an infinite row bound.
template <typename YT>
struct EpiRowKktT {
    const double* __restrict__ row_lo;
    const double* __restrict__ row_hi;
    const YT* __restrict__ y;
    double* __restrict__ part;
    int slot0;
    struct State { double pr2, dr2, dobj, bad; };
    __device__ void init(State& s) const { s.pr2 = s.dr2 = s.dobj = s.bad = 0.0; }
    __device__ void prefetch(int i) const { prefetch_l2(row_lo + i); prefetch_l2(row_hi + i); prefetch_l2(y + i); }
    __device__ void apply(State& s, int i, double act) const {
        const double lo = row_lo[i], hi = row_hi[i];
        if (!isfinite(act)) { s.bad = 1.0; return; }
        const bool lo_f = lo > -1e29, hi_f = hi < 1e29;
        double d = 0.0;
        if (lo_f && act < lo) d = lo - act;
        if (hi_f && act > hi) d = act - hi;
        s.pr2 += d * d;
        const double lam = -static_cast<double>(y[i]);
        if (lam > 0.0) { if (lo_f) s.dobj += lam * lo; else s.dr2 += lam * lam; }
        else if (lam < 0.0) { if (hi_f) s.dobj += lam * hi; else s.dr2 += lam * lam; }
    }
    __device__ void finish(State& s, int channel) const {
        const double v[4] = {s.pr2, s.dr2, s.dobj, s.bad};
        block_sums_to<4>(v, part, channel, slot0);
    }
};

// Column part: reduced cost rc = c + A^T y, the dual objective's bound terms,
// the squared dual infeasibility of an rc sign that pairs with an infinite
// variable bound, the primal objective c^T x, and x's bound violation.
template <typename XT>
struct EpiColKktT {
    const double* __restrict__ c;
    const double* __restrict__ var_lo;
    const double* __restrict__ var_hi;
    const XT* __restrict__ x;
    double* __restrict__ part;
    int slot0;
    struct State { double pr2, dr2, dobj, pobj; };
    __device__ void init(State& s) const { s.pr2 = s.dr2 = s.dobj = s.pobj = 0.0; }
    __device__ void prefetch(int j) const {
        prefetch_l2(c + j); prefetch_l2(var_lo + j); prefetch_l2(var_hi + j); prefetch_l2(x + j);
    }
    __device__ void apply(State& s, int j, double aty) const {
        const double lo = var_lo[j], hi = var_hi[j], cj = c[j];
        const double xj = static_cast<double>(x[j]);
        const bool lo_f = lo > -1e29, hi_f = hi < 1e29;
        const double rc = cj + aty;
        if (rc > 0.0) { if (lo_f) s.dobj += rc * lo; else s.dr2 += rc * rc; }
        else if (rc < 0.0) { if (hi_f) s.dobj += rc * hi; else s.dr2 += rc * rc; }
        s.pobj += cj * xj;
        double d = 0.0;
        if (lo_f && xj < lo) d = lo - xj;
        if (hi_f && xj > hi) d = xj - hi;
        s.pr2 += d * d;
    }
    __device__ void finish(State& s, int channel) const {
        const double v[4] = {s.pr2, s.dr2, s.dobj, s.pobj};
        block_sums_to<4>(v, part, channel, slot0);
    }
};

using EpiRowKkt = EpiRowKktT<float>;     // FP32 iterates
using EpiColKkt = EpiColKktT<float>;
using EpiRowKkt64 = EpiRowKktT<double>;  // FP64 master iterates (refinement)
using EpiColKkt64 = EpiColKktT<double>;

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
