// adaptive_kernels.cuh — element-wise kernels shared by the single-LP and
// batched adaptive PDHG (preconditioning, averaging, restarts, and the FP64
// master / FP32 correction folding of the iterative refinement).
#pragma once

#include "common.cuh"

namespace pb {
namespace {

constexpr int kThreads = 256;
inline int grid_1d(long long n) {
    long long g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    return int(g < 65535LL * 8 ? g : 65535LL * 8);
}

#define PB_GRID_STRIDE(i, n)                                                            \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n);       \
         i += (long long)gridDim.x * blockDim.x)

constexpr double kInf = 1e29;
constexpr float kFltInf = 1e30f;

__global__ void fill_kernel(float* __restrict__ a, int n, float v) {
    PB_GRID_STRIDE(i, n) a[i] = v;
}

// One Ruiz pass over rows (or, run on the transpose, over columns):
// out_scale[i] /= sqrt(max_k |val_k| * in_scale[col_k] * out_scale[i]).
__global__ void ruiz_pass_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                                 const float* __restrict__ val, int rows,
                                 const float* __restrict__ other_scale, float* __restrict__ own_scale,
                                 float* __restrict__ next_scale) {
    PB_GRID_STRIDE(i, rows) {
        const float own = own_scale[i];
        float mx = 0.0f;
        for (int k = rp[i]; k < rp[i + 1]; ++k) mx = fmaxf(mx, fabsf(val[k]) * other_scale[ci[k]]);
        mx *= own;
        next_scale[i] = mx > 0.0f ? own / sqrtf(mx) : own;
    }
}

// Pock-Chambolle (alpha = 1) step of the scaled matrix, mapped back to the
// original variables: step[i] = own[i]^2 / sum_k |val_k| own[i] other[col_k].
__global__ void pc_step_kernel(const int* __restrict__ rp, const int* __restrict__ ci,
                               const float* __restrict__ val, int rows,
                               const float* __restrict__ other_scale, const float* __restrict__ own_scale,
                               float* __restrict__ step) {
    PB_GRID_STRIDE(i, rows) {
        const double own = own_scale[i];
        double s = 0.0;
        for (int k = rp[i]; k < rp[i + 1]; ++k)
            s += fabs(static_cast<double>(val[k])) * static_cast<double>(other_scale[ci[k]]);
        s *= own;
        step[i] = static_cast<float>(s > 1e-30 ? own * own / s : own * own);
    }
}

__global__ void mul_kernel(const float* __restrict__ a, const float* __restrict__ b, int n,
                           float* __restrict__ out) {
    PB_GRID_STRIDE(i, n) out[i] = a[i] * b[i];
}

__global__ void sqrt_kernel(const float* __restrict__ a, int n, float* __restrict__ out) {
    PB_GRID_STRIDE(i, n) out[i] = sqrtf(a[i]);
}

__global__ void scale_kernel(float* __restrict__ a, int n, float s) {
    PB_GRID_STRIDE(i, n) a[i] *= s;
}

__global__ void average_kernel(const double* __restrict__ sum, int n, double inv_count,
                               float* __restrict__ out) {
    PB_GRID_STRIDE(i, n) out[i] = static_cast<float>(sum[i] * inv_count);
}

__global__ void copy2_kernel(const float* __restrict__ src, int n, float* __restrict__ d1,
                             float* __restrict__ d2) {
    PB_GRID_STRIDE(i, n) {
        const float v = src[i];
        d1[i] = v;
        if (d2) d2[i] = v;
    }
}

// Starting master: x_m = clamp(0, l_x, u_x) (the reference's x0), y_m = 0.
// xm = clamp(xw, l, u): the FP64 master iterate of a warm start.
__global__ void init_master_warm_kernel(const double* __restrict__ xw, const double* __restrict__ vlo,
                                        const double* __restrict__ vhi, int n, double* __restrict__ xm) {
    PB_GRID_STRIDE(j, n) {
        double v = xw[j];
        if (vhi[j] < kInf && v > vhi[j]) v = vhi[j];
        if (vlo[j] > -kInf && v < vlo[j]) v = vlo[j];
        xm[j] = v;
    }
}

__global__ void init_master_kernel(const double* __restrict__ vlo, const double* __restrict__ vhi, int n,
                                   double* __restrict__ xm) {
    PB_GRID_STRIDE(j, n) {
        double v = 0.0;
        if (vhi[j] < kInf && v > vhi[j]) v = vhi[j];
        if (vlo[j] > -kInf && v < vlo[j]) v = vlo[j];
        xm[j] = v;
    }
}

// master += correction; correction <- 0 (and the second buffer, if given).
__global__ void fold_into_kernel(double* __restrict__ master, float* __restrict__ corr,
                                 float* __restrict__ corr2, int n) {
    PB_GRID_STRIDE(i, n) {
        master[i] += static_cast<double>(corr[i]);
        corr[i] = 0.0f;
        if (corr2) corr2[i] = 0.0f;
    }
}

// Row data of the correction problem: r_lo = A x_m - l_r, r_hi = A x_m - u_r
// (+1e30 / -1e30 for an infinite bound), and the FP32 copy of y_m.
__global__ void fold_rows_kernel(const double* __restrict__ rlo, const double* __restrict__ rhi,
                                 const double* __restrict__ act, const double* __restrict__ ym, int m,
                                 float* __restrict__ r_lo, float* __restrict__ r_hi, float* __restrict__ ym32) {
    PB_GRID_STRIDE(i, m) {
        const double a = act[i], lo = rlo[i], hi = rhi[i];
        r_lo[i] = lo > -kInf ? static_cast<float>(a - lo) : kFltInf;
        r_hi[i] = hi < kInf ? static_cast<float>(a - hi) : -kFltInf;
        ym32[i] = static_cast<float>(ym[i]);
    }
}

// Column data: rc_m = c + A^T y_m (in place over A^T y_m) and its FP32 copy
// as the correction's cost; bounds l_x - x_m, u_x - x_m.
__global__ void fold_cols_kernel(const double* __restrict__ c, const double* __restrict__ vlo,
                                 const double* __restrict__ vhi, const double* __restrict__ xm, int n,
                                 double* __restrict__ rc, float* __restrict__ c32, float* __restrict__ lx,
                                 float* __restrict__ ux) {
    PB_GRID_STRIDE(j, n) {
        const double r = c[j] + rc[j];
        rc[j] = r;
        c32[j] = static_cast<float>(r);
        const double lo = vlo[j], hi = vhi[j], x = xm[j];
        lx[j] = lo > -kInf ? static_cast<float>(lo - x) : -kFltInf;
        ux[j] = hi < kInf ? static_cast<float>(hi - x) : kFltInf;
    }
}

// out = master + correction in FP64.
__global__ void sum_out_kernel(const double* __restrict__ master, const float* __restrict__ corr, int n,
                               double* __restrict__ out) {
    PB_GRID_STRIDE(i, n) out[i] = master[i] + static_cast<double>(corr[i]);
}

// The original problem's FP32 vectors (as the reference prepares them).
__global__ void restore_cols_kernel(const double* __restrict__ c64, const double* __restrict__ vlo,
                                    const double* __restrict__ vhi, int n, float* __restrict__ c32,
                                    float* __restrict__ flo, float* __restrict__ fhi) {
    PB_GRID_STRIDE(j, n) {
        c32[j] = static_cast<float>(c64[j]);
        flo[j] = vlo[j] <= -kInf ? -kFltInf : static_cast<float>(vlo[j]);
        fhi[j] = vhi[j] >= kInf ? kFltInf : static_cast<float>(vhi[j]);
    }
}

__global__ void restore_rows_kernel(const double* __restrict__ rlo, const double* __restrict__ rhi, int m,
                                    float* __restrict__ flo, float* __restrict__ fhi) {
    PB_GRID_STRIDE(i, m) {
        flo[i] = rlo[i] <= -kInf ? -kFltInf : static_cast<float>(rlo[i]);
        fhi[i] = rhi[i] >= kInf ? kFltInf : static_cast<float>(rhi[i]);
    }
}

}  // namespace
}  // namespace pb
