// epilogues.cuh — per-row epilogues fused into spmv_merge_kernel.
//
// Each epilogue receives a finished row of the product (A x̄ for the dual
// side, Aᵀ y for the primal side) and applies the vector update of the PDHG
// iteration in the same pass, so the product never round-trips through HBM.
#pragma once

#include "spmv.cuh"

namespace pb {

struct NoState {};

// y[r] = value (plain SpMV; test-harness launchers and FP64 row activity).
template <typename AccT, typename OutT>
struct EpiStore {
    OutT* __restrict__ y;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int) const {}
    __device__ void apply(State&, int r, AccT v) const { y[r] = static_cast<OutT>(v); }
    __device__ void finish(State&, int) const {}
};

// Reference dual update with ranged-row projection
// (src/gpu/pdhg_kernels.cuh:72-89):
//   w = y/σ + (A x̄)_i ;  y ← σ (w − clamp(w, l_r, u_r)) ;  rows with σ ≤ 0 untouched.
struct EpiDualRef {
    const float* __restrict__ sigma;
    const float* __restrict__ l_r;
    const float* __restrict__ u_r;
    float* __restrict__ y;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int i) const {
        prefetch_l2(sigma + i); prefetch_l2(l_r + i); prefetch_l2(u_r + i); prefetch_l2(y + i);
    }
    __device__ void apply(State&, int i, float ax) const {
        const float sig = sigma[i];
        if (sig <= 0.0f) return;
        const float w = __fadd_rn(__fdiv_rn(y[i], sig), ax);
        const float wp = fminf(fmaxf(w, l_r[i]), u_r[i]);
        y[i] = __fmul_rn(sig, __fsub_rn(w, wp));
    }
    __device__ void finish(State&, int) const {}
};

// Reference primal update with box projection and extrapolation
// (src/gpu/pdhg_kernels.cuh:95-109):
//   x' = clamp(x − τ (c + Aᵀy), l_x, u_x);  x̄ = 2x' − x;  x = x'.
// The two multiply-adds are written as explicit FMAs: that is what nvcc's
// default contraction produces for the reference expressions.
struct EpiPrimalRef {
    const float* __restrict__ tau;
    const float* __restrict__ c;
    const float* __restrict__ l_x;
    const float* __restrict__ u_x;
    float* __restrict__ x;
    float* __restrict__ x_bar;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int j) const {
        prefetch_l2(tau + j); prefetch_l2(c + j); prefetch_l2(l_x + j); prefetch_l2(u_x + j);
        prefetch_l2(x + j);
    }
    __device__ void apply(State&, int j, float aty) const {
        const float x_prev = x[j];
        const float g = __fadd_rn(c[j], aty);
        const float step = __fmaf_rn(-tau[j], g, x_prev);
        const float x_new = fminf(fmaxf(step, l_x[j]), u_x[j]);
        x_bar[j] = __fmaf_rn(2.0f, x_new, -x_prev);
        x[j] = x_new;
    }
    __device__ void finish(State&, int) const {}
};

// The primal update of a product split in two parts: `add[j]` holds the sum of
// column j's entries from the hot rows of A (the panel part), and the tiled
// product over the other entries passes its own sum; Aᵀy = add[j] + sum.
struct EpiPrimalRefAdd {
    EpiPrimalRef base;
    const float* __restrict__ add;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int j) const {
        base.prefetch(j);
        prefetch_l2(add + j);
    }
    __device__ void apply(State& s, int j, float aty) const { base.apply(s, j, __fadd_rn(add[j], aty)); }
    __device__ void finish(State&, int) const {}
};

// Reductions land in a small device array of doubles:
enum ResidSlot : int {
    kSlotRowViol = 0,     // max row violation  (Ax outside [row_lower, row_upper])
    kSlotBoundViol = 1,   // max bound violation (x outside [var_lower, var_upper])
    kSlotDualViol = 2,    // max projected reduced-cost violation (unnormalised)
    kSlotNonFinite = 3,   // > 0 when a non-finite activity or reduced cost was seen
    kSlotCount = 8
};

// Row part of the reference FP64 residual (src/gpu/pdhg_solver.cu:124-130):
// pv = max over rows of (row_lower − act)+ and (act − row_upper)+ in FP64.
struct EpiRowViolRef {
    const double* __restrict__ row_lo;
    const double* __restrict__ row_hi;
    double* __restrict__ slots;
    struct State { double mx; bool bad; };
    __device__ void init(State& s) const { s.mx = 0.0; s.bad = false; }
    __device__ void prefetch(int i) const { prefetch_l2(row_lo + i); prefetch_l2(row_hi + i); }
    __device__ void apply(State& s, int i, double act) const {
        if (!isfinite(act)) { s.bad = true; return; }
        const double lo = row_lo[i], hi = row_hi[i];
        if (act < lo) s.mx = fmax(s.mx, lo - act);
        if (act > hi) s.mx = fmax(s.mx, act - hi);
    }
    __device__ void finish(State& s, int) const {
        block_max_to(s.mx, &slots[kSlotRowViol]);
        if (s.bad) atomic_max_nonneg(&slots[kSlotNonFinite], 1.0);
    }
};

// Column part of the reference FP64 residual (src/gpu/pdhg_solver.cu:131-157):
// bound violation of x, and the projected reduced-cost violation with rc =
// c + Aᵀy (c and the FP32 matrix values promoted to FP64, as the reference
// does with h_c / h_vl), `tol` slack deciding "at bound".
template <typename XT>
struct EpiColResidRefT {
    const XT* __restrict__ x;
    const float* __restrict__ c;
    const double* __restrict__ var_lo;
    const double* __restrict__ var_hi;
    double tol;
    double* __restrict__ slots;
    struct State { double bmx, dmx; bool bad; };
    __device__ void init(State& s) const { s.bmx = 0.0; s.dmx = 0.0; s.bad = false; }
    __device__ void prefetch(int j) const {
        prefetch_l2(x + j); prefetch_l2(c + j); prefetch_l2(var_lo + j); prefetch_l2(var_hi + j);
    }
    __device__ void apply(State& s, int j, double aty) const {
        const double xd = static_cast<double>(x[j]);
        const double lo = var_lo[j], hi = var_hi[j];
        if (!isfinite(xd) || !isfinite(aty)) { s.bad = true; return; }
        if (xd < lo) s.bmx = fmax(s.bmx, lo - xd);
        if (xd > hi) s.bmx = fmax(s.bmx, xd - hi);
        const double rc = static_cast<double>(c[j]) + aty;
        const bool at_lb = xd <= lo + tol;
        const bool at_ub = xd >= hi - tol;
        double viol = 0.0;
        if (!at_lb && !at_ub) viol = fabs(rc);
        else if (at_lb && !at_ub) viol = fmax(0.0, -rc);
        else if (at_ub && !at_lb) viol = fmax(0.0, rc);
        s.dmx = fmax(s.dmx, viol);
    }
    __device__ void finish(State& s, int) const {
        block_max_to(s.bmx, &slots[kSlotBoundViol]);
        block_max_to(s.dmx, &slots[kSlotDualViol]);
        if (s.bad) atomic_max_nonneg(&slots[kSlotNonFinite], 1.0);
    }
};
using EpiColResidRef = EpiColResidRefT<float>;

}  // namespace pb
