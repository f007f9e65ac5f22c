// pdhg_refine.cu — FP64 iterative refinement on the GPU (adaptive mode,
// refine_rounds > 0).
//
// The FP32 iteration resolves the relative KKT error to about 1e-7.  To
// reach 1e-8 the solver keeps FP64 master iterates (x, y) on the device and
// repeats, after Gleixner, Steffy and Wolter ("Iterative refinement for
// linear programming", INFORMS J. Computing 2016):
//   1. in FP64: act = A x, rc = c + A^T y (the reduced cost in the reference's
//      sign convention, y the negated multiplier), the largest primal
//      violation dP and the largest dual infeasibility dD;
//   2. scale factors SP = 1/dP, SD = 1/dD (each at most 1e6 times the previous
//      round's and at most 1e14);
//   3. the correction LP with the same matrix:
//        min (SD rc)^T d   s.t.  SP (l_r - act) <= A d <= SP (u_r - act),
//                                SP (l_x - x)   <=  d  <= SP (u_x - x),
//      solved by the FP32 adaptive iteration to `tolerance` (relative KKT),
//      from d = clamp(0), y = 0;
//   4. x += d / SP, y += y_corr / SD in FP64,
// until the relative KKT error of (x, y) on the original problem is at most
// refine_tolerance or refine_rounds rounds have run.  Only vectors change
// between rounds; the matrix, its tile records, the preconditioned steps and
// the step size are reused.
#include "adaptive.cuh"
#include "pdhg_engine.cuh"

#include <cmath>
#include <limits>

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

__global__ void to_double_kernel(const float* __restrict__ a, int n, double* __restrict__ out) {
    PB_GRID_STRIDE(i, n) out[i] = static_cast<double>(a[i]);
}

// Largest primal violation (rows and bounds) and largest dual infeasibility
// (reduced costs and multipliers whose sign pairs with an infinite bound).
__global__ void infeasibility_kernel(const double* __restrict__ act, const double* __restrict__ rlo,
                                     const double* __restrict__ rhi, const double* __restrict__ y,
                                     int m, const double* __restrict__ x, const double* __restrict__ vlo,
                                     const double* __restrict__ vhi, const double* __restrict__ rc, int n,
                                     double* __restrict__ out) {
    double pmax = 0.0, dmax = 0.0;
    PB_GRID_STRIDE(i, (long long)m + n) {
        if (i < m) {
            const double a = act[i], lo = rlo[i], hi = rhi[i];
            if (lo > -kInf && a < lo) pmax = fmax(pmax, lo - a);
            if (hi < kInf && a > hi) pmax = fmax(pmax, a - hi);
            const double lam = -y[i];
            if (lam > 0.0 && !(lo > -kInf)) dmax = fmax(dmax, lam);
            if (lam < 0.0 && !(hi < kInf)) dmax = fmax(dmax, -lam);
        } else {
            const long long j = i - m;
            const double xj = x[j], lo = vlo[j], hi = vhi[j], r = rc[j];
            if (lo > -kInf && xj < lo) pmax = fmax(pmax, lo - xj);
            if (hi < kInf && xj > hi) pmax = fmax(pmax, xj - hi);
            if (r > 0.0 && !(lo > -kInf)) dmax = fmax(dmax, r);
            if (r < 0.0 && !(hi < kInf)) dmax = fmax(dmax, -r);
        }
    }
    block_max_to(pmax, &out[0]);
    block_max_to(dmax, &out[1]);
}

// Correction LP, row side: SP (l_r - act) .. SP (u_r - act) in FP64 and FP32
// (infinite bounds stay infinite); y_corr starts at 0.
__global__ void corr_rows_kernel(const double* __restrict__ rlo, const double* __restrict__ rhi,
                                 const double* __restrict__ act, int m, double sp,
                                 double* __restrict__ clo, double* __restrict__ chi, float* __restrict__ flo,
                                 float* __restrict__ fhi, float* __restrict__ y32) {
    PB_GRID_STRIDE(i, m) {
        const double lo = rlo[i], hi = rhi[i], a = act[i];
        const double l = lo > -kInf ? sp * (lo - a) : -1e30;
        const double h = hi < kInf ? sp * (hi - a) : 1e30;
        clo[i] = l;
        chi[i] = h;
        flo[i] = l <= -kInf ? -kFltInf : static_cast<float>(l);
        fhi[i] = h >= kInf ? kFltInf : static_cast<float>(h);
        y32[i] = 0.0f;
    }
}

// Correction LP, column side: cost SD rc, bounds SP (l_x - x) .. SP (u_x - x);
// d starts at clamp(0, lower, upper).
__global__ void corr_cols_kernel(const double* __restrict__ vlo, const double* __restrict__ vhi,
                                 const double* __restrict__ x, const double* __restrict__ rc, int n,
                                 double sp, double sd, double* __restrict__ cc, double* __restrict__ clo,
                                 double* __restrict__ chi, float* __restrict__ c32, float* __restrict__ flo,
                                 float* __restrict__ fhi, float* __restrict__ x32, float* __restrict__ xbar) {
    PB_GRID_STRIDE(j, n) {
        const double lo = vlo[j], hi = vhi[j], xj = x[j];
        const double l = lo > -kInf ? sp * (lo - xj) : -1e30;
        const double h = hi < kInf ? sp * (hi - xj) : 1e30;
        const double c = sd * rc[j];
        cc[j] = c;
        clo[j] = l;
        chi[j] = h;
        c32[j] = static_cast<float>(c);
        const float fl = l <= -kInf ? -kFltInf : static_cast<float>(l);
        const float fh = h >= kInf ? kFltInf : static_cast<float>(h);
        flo[j] = fl;
        fhi[j] = fh;
        const float d0 = fmaxf(fl, fminf(0.0f, fh));
        x32[j] = d0;
        xbar[j] = d0;
    }
}

// master += correction / scale
__global__ void master_update_kernel(double* __restrict__ master, const float* __restrict__ corr, int n,
                                     double inv_scale) {
    PB_GRID_STRIDE(i, n) master[i] += static_cast<double>(corr[i]) * inv_scale;
}

__global__ void add_kernel(const double* __restrict__ a, const double* __restrict__ b, int n,
                           double* __restrict__ out) {
    PB_GRID_STRIDE(i, n) out[i] = a[i] + b[i];
}

// Original problem's FP32 vectors again (for the FP32 fields of the result).
__global__ void restore_kernel(const double* __restrict__ c64, const double* __restrict__ vlo,
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

// Deterministic FP64 sum of squares of finite bound entries (norm of b of the
// correction problem) and of a vector (norm of its cost).
__global__ void norms_kernel(const double* __restrict__ lo, const double* __restrict__ hi, int m,
                             const double* __restrict__ c, int n, double* __restrict__ part) {
    double b2 = 0.0, c2 = 0.0;
    PB_GRID_STRIDE(i, (long long)m + n) {
        if (i < m) {
            const double l = lo[i], h = hi[i];
            if (l > -kInf) b2 += l * l;
            if (h < kInf && !(l > -kInf && l == h)) b2 += h * h;
        } else {
            const double v = c[i - m];
            c2 += v * v;
        }
    }
    const double v[2] = {b2, c2};
    block_sums_to<2>(v, part, 0, 0);
}

__global__ void reduce2_kernel(const double* __restrict__ part, int rows, double* __restrict__ out) {
    __shared__ double s0[256], s1[256];
    double a = 0.0, b = 0.0;
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
        a += part[size_t(r) * kPartSlots + 0];
        b += part[size_t(r) * kPartSlots + 1];
    }
    s0[threadIdx.x] = a;
    s1[threadIdx.x] = b;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) { s0[threadIdx.x] += s0[threadIdx.x + w]; s1[threadIdx.x] += s1[threadIdx.x + w]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = s0[0]; out[1] = s1[0]; }
}

}  // namespace

void PdhgEngine::refine(pramaan_solve_result* res) {
    refined_ = true;
    x64_.alloc(n_); y64_.alloc(m_); act64_.alloc(m_); aty64_.alloc(n_);
    cc64_.alloc(n_); cvlo64_.alloc(n_); cvhi64_.alloc(n_); crlo64_.alloc(m_); crhi64_.alloc(m_);
    if (n_) to_double_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x_.get(), n_, x64_.get());
    if (m_) to_double_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(y_.get(), m_, y64_.get());
    PB_CUDA_CHECK(cudaGetLastError());

    const double target = opt_.refine_tolerance;
    double sp_prev = 1.0, sd_prev = 1.0;
    Kkt k;
    int status = res->status;
    for (int round = 0; round < opt_.refine_rounds; ++round) {
        kkt_master(k);
        if (k.nonfinite) { status = PRAMAAN_STATUS_NUMERICAL_FAILURE; break; }
        if (k.converged(target)) { status = PRAMAAN_STATUS_OPTIMAL; break; }
        // FP64 residuals of the master iterate
        if (m_) {
            EpiStore<double, double> e{act64_.get()};
            if (A_.has_lo)
                SpmvLauncher<EpiStore<double, double>, double, double, true>::launch(A_.view(true), x64_.get(), e, status_.get(), st_, dev_);
            else
                SpmvLauncher<EpiStore<double, double>, double, double, false>::launch(A_.view(false), x64_.get(), e, status_.get(), st_, dev_);
        }
        if (n_) {
            EpiStore<double, double> e{aty64_.get()};
            if (AT_.has_lo)
                SpmvLauncher<EpiStore<double, double>, double, double, true>::launch(AT_.view(true), y64_.get(), e, status_.get(), st_, dev_);
            else
                SpmvLauncher<EpiStore<double, double>, double, double, false>::launch(AT_.view(false), y64_.get(), e, status_.get(), st_, dev_);
            add_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cmin64_.get(), aty64_.get(), n_, aty64_.get());   // rc
            PB_CUDA_CHECK(cudaGetLastError());
        }
        PB_CUDA_CHECK(cudaMemsetAsync(slots_.get(), 0, sizeof(double) * kSlotCount, st_));
        infeasibility_kernel<<<grid_1d((long long)m_ + n_) < 1024 ? grid_1d((long long)m_ + n_) : 1024, kThreads, 0, st_>>>(
            act64_.get(), rlo64_.get(), rhi64_.get(), y64_.get(), m_, x64_.get(), vlo64_.get(), vhi64_.get(),
            aty64_.get(), n_, slots_.get());
        PB_CUDA_CHECK(cudaGetLastError());
        PB_CUDA_CHECK(cudaMemcpyAsync(h_slots_, slots_.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        const double dP = h_slots_[0], dD = h_slots_[1];
        // the complementarity part is carried by the objective gap of the correction LP
        double sp = dP > 1e-300 ? 1.0 / dP : 1e14;
        double sd = dD > 1e-300 ? 1.0 / dD : 1e14;
        sp = std::min(std::min(sp, 1e14), 1e6 * sp_prev);
        sd = std::min(std::min(sd, 1e14), 1e6 * sd_prev);
        sp = std::max(sp, 1.0);
        sd = std::max(sd, 1.0);
        sp_prev = sp;
        sd_prev = sd;
        // correction problem
        if (m_) corr_rows_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rlo64_.get(), rhi64_.get(), act64_.get(), m_, sp,
                                                                    crlo64_.get(), crhi64_.get(), lr_.get(), ur_.get(), y_.get());
        if (n_) corr_cols_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(vlo64_.get(), vhi64_.get(), x64_.get(), aty64_.get(),
                                                                    n_, sp, sd, cc64_.get(), cvlo64_.get(), cvhi64_.get(),
                                                                    c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get());
        PB_CUDA_CHECK(cudaGetLastError());
        pc64_ = cc64_.get();
        prlo_ = crlo64_.get();
        prhi_ = crhi64_.get();
        pvlo_ = cvlo64_.get();
        pvhi_ = cvhi64_.get();
        PB_CUDA_CHECK(cudaMemsetAsync(part_.get(), 0, part_.bytes(), st_));
        norms_kernel<<<256, kThreads, 0, st_>>>(prlo_, prhi_, m_, pc64_, n_, part_.get());
        reduce2_kernel<<<1, 256, 0, st_>>>(part_.get(), kPartRows, red_.get());
        PB_CUDA_CHECK(cudaGetLastError());
        PB_CUDA_CHECK(cudaMemcpyAsync(h_red_, red_.get(), 16, cudaMemcpyDeviceToHost, st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        pb_norm_ = std::sqrt(h_red_[0]);
        pc_norm_ = std::sqrt(h_red_[1]);
        restart_to(false);
        const int st = adaptive_loop(opt_.tolerance, opt_.max_iterations, res, nullptr);
        if (st == PRAMAAN_STATUS_NUMERICAL_FAILURE) { status = st; break; }
        if (n_) master_update_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x64_.get(), x_.get(), n_, 1.0 / sp);
        if (m_) master_update_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(y64_.get(), y_.get(), m_, 1.0 / sd);
        PB_CUDA_CHECK(cudaGetLastError());
        status = PRAMAAN_STATUS_ITERATION_LIMIT;
    }
    if (status != PRAMAAN_STATUS_NUMERICAL_FAILURE) {
        kkt_master(k);
        status = k.converged(target) ? PRAMAAN_STATUS_OPTIMAL : PRAMAAN_STATUS_ITERATION_LIMIT;
    }
    // back to the original problem's vectors
    use_original_problem();
    if (n_) restore_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cmin64_.get(), vlo64_.get(), vhi64_.get(), n_,
                                                               c_.get(), lx_.get(), ux_.get());
    if (m_) restore_rows_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rlo64_.get(), rhi64_.get(), m_, lr_.get(), ur_.get());
    PB_CUDA_CHECK(cudaGetLastError());
    res->status = status;
    res->iterations = total_iterations_;
    res->rel_primal = k.rel_p;
    res->rel_dual = k.rel_d;
    res->rel_gap = k.rel_gap;
}

}  // namespace pb
