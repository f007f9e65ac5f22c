// batch.cu — AdaptiveBatch: many LPs in one packed operand (see batch.cuh).
#include "batch.cuh"

#include "adaptive.cuh"
#include "adaptive_kernels.cuh"
#include "cluster_interval.cuh"
#include "interval.cuh"
#include "pdhg_engine.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <limits>

namespace pb {

namespace {

constexpr int kChunk = 4096;       // elements per reduction chunk (never straddles two LPs)
constexpr int kOutWidth = 16;      // doubles per LP in the reduction output

enum : int {
    kActNone = 0,
    kActRestartCurrent = 1,   // restart from the current iterate (then fold / record)
    kActRestartAverage = 2,   // restart from the average (then fold / record)
    kActFreezeAverage = 3,    // converged on the average: take it, no fold
};

// ---- per-LP reductions ---------------------------------------------------

// One block per chunk: sums (or maxima) of `width` <= 4 interleaved values.
template <bool kMax>
__global__ void chunk_reduce_kernel(const double* __restrict__ contrib, int width,
                                    const int* __restrict__ begin, double* __restrict__ out) {
    __shared__ double sh[4][256];
    const int c = blockIdx.x;
    const int b = begin[c], e = begin[c + 1];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = b + threadIdx.x; i < e; i += blockDim.x)
        for (int s = 0; s < width; ++s) {
            const double v = contrib[size_t(i) * width + s];
            acc[s] = kMax ? fmax(acc[s], v) : acc[s] + v;
        }
    for (int s = 0; s < width; ++s) sh[s][threadIdx.x] = acc[s];
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            for (int s = 0; s < width; ++s) {
                const double a = sh[s][threadIdx.x], o = sh[s][threadIdx.x + w];
                sh[s][threadIdx.x] = kMax ? fmax(a, o) : a + o;
            }
        __syncthreads();
    }
    if (threadIdx.x < width) out[size_t(c) * width + threadIdx.x] = sh[threadIdx.x][0];
}

// One thread per (LP, slot): the LP's chunks in order.
template <bool kMax>
__global__ void lp_reduce_kernel(const double* __restrict__ chunk_out, int width,
                                 const int* __restrict__ lp_first, int K, double* __restrict__ out,
                                 int out_off) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= K * width) return;
    const int k = t / width, s = t % width;
    double acc = 0.0;
    for (int c = lp_first[k]; c < lp_first[k + 1]; ++c) {
        const double v = chunk_out[size_t(c) * width + s];
        acc = kMax ? fmax(acc, v) : acc + v;
    }
    out[size_t(k) * kOutWidth + out_off + s] = acc;
}

// ---- per-element epilogues writing contributions ---------------------------

// Relative-KKT row terms of x = x_m + d, y = y_m + e (as EpiRowKkt), one
// 4-tuple per row: pr2, dr2, dobj, non-finite flag.
struct EpiRowKktOut {
    const double* __restrict__ row_lo;
    const double* __restrict__ row_hi;
    const double* __restrict__ act_m;
    const double* __restrict__ y_m;
    const float* __restrict__ e;
    double* __restrict__ out;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int i) const {
        prefetch_l2(row_lo + i); prefetch_l2(row_hi + i); prefetch_l2(act_m + i); prefetch_l2(y_m + i);
        prefetch_l2(e + i);
    }
    __device__ void apply(State&, int i, double ad) const {
        double* o = out + size_t(i) * 4;
        const double lo = row_lo[i], hi = row_hi[i];
        const double act = act_m[i] + ad;
        if (!isfinite(act)) { o[0] = 0.0; o[1] = 0.0; o[2] = 0.0; o[3] = 1.0; return; }
        const bool lo_f = lo > -1e29, hi_f = hi < 1e29;
        double d = 0.0;
        if (lo_f && act < lo) d = lo - act;
        if (hi_f && act > hi) d = act - hi;
        double dr2 = 0.0, dobj = 0.0;
        const double lam = -(y_m[i] + static_cast<double>(e[i]));
        if (lam > 0.0) { if (lo_f) dobj = lam * lo; else dr2 = lam * lam; }
        else if (lam < 0.0) { if (hi_f) dobj = lam * hi; else dr2 = lam * lam; }
        o[0] = d * d; o[1] = dr2; o[2] = dobj; o[3] = 0.0;
    }
    __device__ void finish(State&, int) const {}
};

// Relative-KKT column terms (as EpiColKkt): pr2 (bound violation), dr2, dobj, pobj.
struct EpiColKktOut {
    const double* __restrict__ c;
    const double* __restrict__ var_lo;
    const double* __restrict__ var_hi;
    const double* __restrict__ rc_m;
    const double* __restrict__ x_m;
    const float* __restrict__ d;
    double* __restrict__ out;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int j) const {
        prefetch_l2(c + j); prefetch_l2(var_lo + j); prefetch_l2(var_hi + j); prefetch_l2(rc_m + j);
        prefetch_l2(x_m + j); prefetch_l2(d + j);
    }
    __device__ void apply(State&, int j, double ate) const {
        double* o = out + size_t(j) * 4;
        const double lo = var_lo[j], hi = var_hi[j], cj = c[j];
        const double xj = x_m[j] + static_cast<double>(d[j]);
        const bool lo_f = lo > -1e29, hi_f = hi < 1e29;
        const double rc = rc_m[j] + ate;
        double dr2 = 0.0, dobj = 0.0;
        if (rc > 0.0) { if (lo_f) dobj = rc * lo; else dr2 = rc * rc; }
        else if (rc < 0.0) { if (hi_f) dobj = rc * hi; else dr2 = rc * rc; }
        double v = 0.0;
        if (lo_f && xj < lo) v = lo - xj;
        if (hi_f && xj > hi) v = xj - hi;
        o[0] = v * v; o[1] = dr2; o[2] = dobj; o[3] = cj * xj;
    }
    __device__ void finish(State&, int) const {}
};

// Reference criterion (src/gpu/pdhg_solver.cu:124-130), per row: violation, non-finite flag.
struct EpiRowViolOut {
    const double* __restrict__ row_lo;
    const double* __restrict__ row_hi;
    double* __restrict__ out;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int i) const { prefetch_l2(row_lo + i); prefetch_l2(row_hi + i); }
    __device__ void apply(State&, int i, double act) const {
        double* o = out + size_t(i) * 2;
        if (!isfinite(act)) { o[0] = 0.0; o[1] = 1.0; return; }
        double v = 0.0;
        if (act < row_lo[i]) v = row_lo[i] - act;
        if (act > row_hi[i]) v = fmax(v, act - row_hi[i]);
        o[0] = v; o[1] = 0.0;
    }
    __device__ void finish(State&, int) const {}
};

// Reference criterion (src/gpu/pdhg_solver.cu:131-157), per column: bound
// violation, projected reduced-cost violation (FP32 c promoted, `tol` slack),
// non-finite flag.
struct EpiColResidOut {
    const double* __restrict__ x;
    const float* __restrict__ c;
    const double* __restrict__ var_lo;
    const double* __restrict__ var_hi;
    double tol;
    double* __restrict__ out;
    using State = NoState;
    __device__ void init(State&) const {}
    __device__ void prefetch(int j) const {
        prefetch_l2(x + j); prefetch_l2(c + j); prefetch_l2(var_lo + j); prefetch_l2(var_hi + j);
    }
    __device__ void apply(State&, int j, double aty) const {
        double* o = out + size_t(j) * 3;
        const double xd = x[j], lo = var_lo[j], hi = var_hi[j];
        if (!isfinite(xd) || !isfinite(aty)) { o[0] = 0.0; o[1] = 0.0; o[2] = 1.0; return; }
        double b = 0.0;
        if (xd < lo) b = lo - xd;
        if (xd > hi) b = fmax(b, xd - hi);
        const double rc = static_cast<double>(c[j]) + aty;
        const bool at_lb = xd <= lo + tol;
        const bool at_ub = xd >= hi - tol;
        double viol = 0.0;
        if (!at_lb && !at_ub) viol = fabs(rc);
        else if (at_lb && !at_ub) viol = fmax(0.0, -rc);
        else if (at_ub && !at_lb) viol = fmax(0.0, rc);
        o[0] = b; o[1] = viol; o[2] = 0.0;
    }
    __device__ void finish(State&, int) const {}
};

// ---- per-LP element-wise kernels ------------------------------------------

__global__ void scale_steps_kernel(const float* __restrict__ base, const int* __restrict__ lp,
                                   const float* __restrict__ scale, int len, float* __restrict__ eff) {
    PB_GRID_STRIDE(i, len) eff[i] = base[i] * scale[lp[i]];
}

// out = sum * inv[lp]; an LP with inv < 0 has no averaged iterations yet: out = cur.
__global__ void average_lp_kernel(const double* __restrict__ sum, const float* __restrict__ cur,
                                  const int* __restrict__ lp, const double* __restrict__ inv, int len,
                                  float* __restrict__ out) {
    PB_GRID_STRIDE(i, len) {
        const double f = inv[lp[i]];
        out[i] = f < 0.0 ? cur[i] : static_cast<float>(sum[i] * f);
    }
}

// Restart of the LPs with an action: from the average for kActRestartAverage
// and kActFreezeAverage; extrapolated iterate reset; epoch sums cleared.
__global__ void restart_lp_kernel(const int* __restrict__ lp, const int* __restrict__ action, int len,
                                  float* __restrict__ v, const float* __restrict__ avg,
                                  float* __restrict__ vbar, double* __restrict__ sum) {
    PB_GRID_STRIDE(i, len) {
        const int a = action[lp[i]];
        if (a == kActNone) continue;
        if (a == kActRestartAverage || a == kActFreezeAverage) v[i] = avg[i];
        if (vbar) vbar[i] = v[i];
        sum[i] = 0.0;
    }
}

// FP64 refinement fold of the restarting LPs: master += correction, correction <- 0.
__global__ void fold_lp_kernel(const int* __restrict__ lp, const int* __restrict__ action, int len,
                               double* __restrict__ master, float* __restrict__ corr,
                               float* __restrict__ corr2) {
    PB_GRID_STRIDE(i, len) {
        const int a = action[lp[i]];
        if (a != kActRestartCurrent && a != kActRestartAverage) continue;
        master[i] += static_cast<double>(corr[i]);
        corr[i] = 0.0f;
        if (corr2) corr2[i] = 0.0f;
    }
}

// Restart point of the restarting LPs (plain FP32 iterates, refine = 0).
__global__ void record_lp_kernel(const int* __restrict__ lp, const int* __restrict__ action, int len,
                                 const float* __restrict__ src, float* __restrict__ dst) {
    PB_GRID_STRIDE(i, len) {
        const int a = action[lp[i]];
        if (a == kActRestartCurrent || a == kActRestartAverage) dst[i] = src[i];
    }
}

// ((a - sub) / scale)^2 per element (sub may be null).
__global__ void dist_contrib_kernel(const float* __restrict__ a, const float* __restrict__ sub,
                                    const float* __restrict__ scale, int len, double* __restrict__ out) {
    PB_GRID_STRIDE(i, len) {
        double u = static_cast<double>(a[i]) - (sub ? static_cast<double>(sub[i]) : 0.0);
        u /= static_cast<double>(scale[i]);
        out[i] = u * u;
    }
}

// Power iteration terms per element: v w and w w.
__global__ void dot2_contrib_kernel(const float* __restrict__ v, const float* __restrict__ w, int len,
                                    double* __restrict__ out) {
    PB_GRID_STRIDE(i, len) {
        const double a = v[i], b = w[i];
        out[2 * i] = a * b;
        out[2 * i + 1] = b * b;
    }
}

__global__ void scale_lp_kernel(const float* __restrict__ w, const int* __restrict__ lp,
                                const float* __restrict__ f, int len, float* __restrict__ v) {
    PB_GRID_STRIDE(i, len) v[i] = w[i] * f[lp[i]];
}

__global__ void fill_lp_kernel(float* __restrict__ v, const int* __restrict__ lp, const float* __restrict__ f,
                               int len) {
    PB_GRID_STRIDE(i, len) v[i] = f[lp[i]];
}

template <typename T>
__global__ void gather_kernel(const T* __restrict__ src, const int* __restrict__ idx, int len, T* __restrict__ dst) {
    PB_GRID_STRIDE(i, len) dst[i] = src[idx[i]];
}

// Answers of the LPs leaving the operand (keep[lp] == 0; every LP when keep
// is null): out[orig(i)] = master[i] + correction[i].
__global__ void scatter_answers_kernel(const int* __restrict__ lp, const int* __restrict__ keep,
                                       const double* __restrict__ master, const float* __restrict__ corr,
                                       const int* __restrict__ orig, int len, double* __restrict__ out) {
    PB_GRID_STRIDE(i, len) {
        if (keep && keep[lp[i]]) continue;
        out[orig ? orig[i] : i] = master[i] + static_cast<double>(corr[i]);
    }
}

__global__ void set_int_kernel(int* p, int v) { *p = v; }

template <typename T>
void regather(DevBuf<T>& b, const DevBuf<int>& map, int len, cudaStream_t st) {
    if (b.size() == 0) return;
    DevBuf<T> nb(static_cast<size_t>(len > 0 ? len : 1));
    if (len > 0) {
        gather_kernel<T><<<grid_1d(len), kThreads, 0, st>>>(b.get(), map.get(), len, nb.get());
        PB_CUDA_CHECK(cudaGetLastError());
    }
    b = std::move(nb);
}

template <typename T>
void copy_buf(DevBuf<T>& dst, const DevBuf<T>& src, cudaStream_t st) {
    dst.alloc(src.size());
    if (src.size())
        PB_CUDA_CHECK(cudaMemcpyAsync(dst.get(), src.get(), src.bytes(), cudaMemcpyDeviceToDevice, st));
}

template <typename Epi, typename AccT, typename XT>
void launch_any(const CsrDevice& A, const XT* x, const Epi& e, int* status, cudaStream_t st, int dev) {
    if (A.has_lo)
        SpmvLauncher<Epi, AccT, XT, true>::launch(A.view(true), x, e, status, st, dev);
    else
        SpmvLauncher<Epi, AccT, XT, false>::launch(A.view(false), x, e, status, st, dev);
}

template <typename Epi, typename AccT, typename XT>
void warm_launcher(int dev) {
    SpmvLauncher<Epi, AccT, XT, true>::blocks_per_sm(dev);
    SpmvLauncher<Epi, AccT, XT, false>::blocks_per_sm(dev);
}

// Cooperative-launch helpers for halpern_interval_kernel.
template <bool kMapA, bool kMapAT>
int interval_blocks_per_sm(int dev) {
    static std::atomic<int> cache[64];
    if (dev < 0 || dev >= 64) dev = 0;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    using L = SpmvSmemLayout<kSpmvWarps, kSpmvStages, false, float>;
    auto k = &halpern_interval_kernel<kMapA, kMapAT>;
    PB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::bytes)));
    int nb = 0;
    PB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kSpmvWarps * 32, L::bytes));
    if (nb < 1) nb = 1;
    cache[dev].store(nb, std::memory_order_relaxed);
    return nb;
}

int interval_bps(bool map_a, bool map_at, int dev) {
    if (map_a) return map_at ? interval_blocks_per_sm<true, true>(dev) : interval_blocks_per_sm<true, false>(dev);
    return map_at ? interval_blocks_per_sm<false, true>(dev) : interval_blocks_per_sm<false, false>(dev);
}

double weighted(double pr2, double dr2, double gap, double omega) {
    return std::sqrt(omega * omega * pr2 + dr2 / (omega * omega) + gap * gap);
}

}  // namespace

AdaptiveBatch::AdaptiveBatch(const pramaan_lp* lps, int count, const pramaan_pdhg_options& opt,
                             const pramaan_warm_start* warm)
    : opt_(opt) {
    validate_options(opt);
    if (opt.algorithm != PRAMAAN_ALGO_ADAPTIVE && opt.algorithm != PRAMAAN_ALGO_HALPERN)
        throw InvalidArgument("batched solves use the adaptive or the Halpern algorithm "
                              "(PRAMAAN_ALGO_ADAPTIVE, PRAMAAN_ALGO_HALPERN)");
    halpern_ = opt.algorithm == PRAMAAN_ALGO_HALPERN;
    if (count < 0) throw InvalidArgument("batch: count must be >= 0");
    dev_ = opt.device;
    count_ = count;
    long long m = 0, n = 0, nnz = 0;
    for (int k = 0; k < count; ++k) {
        const pramaan_lp& lp = lps[k];
        validate_lp(lp);
        if (lp.num_cols == 0) continue;                      // answered without the GPU
        bool finite = true;
        for (int j = 0; j < lp.num_cols; ++j) finite = finite && std::isfinite(lp.obj_coeffs[j]);
        if (!finite) continue;                               // numerical failure, as the reference
        Lp s;
        s.index = k;
        s.r0 = int(m); s.c0 = int(n);
        m += lp.num_rows; n += lp.num_cols; nnz += lp.nnz;
        if (m > INT_MAX / 2 || n > INT_MAX / 2 || nnz > INT_MAX / 2)
            throw InvalidArgument("batch: the packed LP exceeds 2^30 rows, columns or non-zeros");
        s.r1 = int(m); s.c1 = int(n);
        s.or0 = s.r0; s.or1 = s.r1; s.oc0 = s.c0; s.oc1 = s.c1;
        s.nnz = lp.nnz;
        lp_.push_back(s);
    }
    K_ = int(lp_.size());
    m_ = int(m); n_ = int(n); nnz_ = int(nnz);
    full_m_ = m_; full_n_ = n_;
    PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    PB_CUDA_CHECK(pinned_alloc(&h_status_, sizeof(int)));
    status_.alloc(1);
    PB_CUDA_CHECK(cudaMemsetAsync(status_.get(), 0, sizeof(int), st_));
    if (K_ == 0) return;

    // ---- pack the LPs (host), minimisation form ----
    const size_t M = static_cast<size_t>(m_), N = static_cast<size_t>(n_), NZ = static_cast<size_t>(nnz_);
    std::vector<int> rp(M + 1), ci(NZ), lp_row(M), lp_col(N);
    std::vector<double> val(NZ), rl(M), ru(M), vl(N), vu(N), cmin(N);
    std::vector<int> rseg(static_cast<size_t>(K_) + 1), cseg(static_cast<size_t>(K_) + 1);
    long long e0 = 0;
    for (int q = 0; q < K_; ++q) {
        Lp& s = lp_[q];
        const pramaan_lp& lp = lps[s.index];
        const double sign = lp.obj_sense == PRAMAAN_MAXIMIZE ? -1.0 : 1.0;
        double c2 = 0.0, cinf = 1.0;
        for (int j = 0; j < lp.num_cols; ++j) {
            const double cj = sign * lp.obj_coeffs[j];
            cmin[s.c0 + j] = cj;
            c2 += cj * cj;
            cinf = std::max(cinf, double(std::fabs(static_cast<float>(cj))));
            vl[s.c0 + j] = lp.var_lower[j];
            vu[s.c0 + j] = lp.var_upper[j];
            lp_col[s.c0 + j] = q;
        }
        s.c_norm = std::sqrt(c2);
        s.c32_inf = cinf;
        double b2 = 0.0;
        for (int i = 0; i < lp.num_rows; ++i) {
            const double lo = lp.row_lower[i], hi = lp.row_upper[i];
            rl[s.r0 + i] = lo;
            ru[s.r0 + i] = hi;
            if (lo > -1e29) b2 += lo * lo;
            if (hi < 1e29 && !(lo > -1e29 && lo == hi)) b2 += hi * hi;
            lp_row[s.r0 + i] = q;
            rp[s.r0 + i] = int(e0 + lp.row_ptr[i]);
        }
        s.b_norm = std::sqrt(b2);
        for (int k = 0; k < lp.nnz; ++k) {
            ci[e0 + k] = lp.col_idx[k] + s.c0;
            val[e0 + k] = lp.values[k];
        }
        e0 += lp.nnz;
        rseg[q] = s.r0; cseg[q] = s.c0;
    }
    rp[m_] = int(e0);
    rseg[K_] = m_; cseg[K_] = n_;
    std::vector<double> xw, yw;
    if (warm) {
        xw.assign(N, 0.0);
        yw.assign(M, 0.0);
        for (int q = 0; q < K_; ++q) {
            const Lp& s = lp_[q];
            const pramaan_warm_start& w = warm[s.index];
            const int nk = s.c1 - s.c0, mk = s.r1 - s.r0;
            for (int j = 0; j < nk; ++j) {
                const double v = w.x ? w.x[j] : 0.0;
                if (!std::isfinite(v)) throw InvalidArgument("warm start: x must be finite");
                xw[size_t(s.c0 + j)] = v;
            }
            for (int i = 0; i < mk; ++i) {
                const double v = w.y ? w.y[i] : 0.0;
                if (!std::isfinite(v)) throw InvalidArgument("warm start: y must be finite");
                yw[size_t(s.r0 + i)] = v;
            }
        }
    }

    PB_CUDA_CHECK(pinned_alloc(&h_action_, sizeof(int) * K_));
    PB_CUDA_CHECK(pinned_alloc(&h_inv_, sizeof(double) * K_));
    PB_CUDA_CHECK(pinned_alloc(&h_dscale_, sizeof(float) * K_));
    PB_CUDA_CHECK(pinned_alloc(&h_pscale_, sizeof(float) * K_));
    PB_CUDA_CHECK(pinned_alloc(&h_lp_f_, sizeof(float) * K_));
    PB_CUDA_CHECK(pinned_alloc(&h_out_, sizeof(double) * K_ * kOutWidth));
    PB_CUDA_CHECK(pinned_alloc(&h_keep_, sizeof(int) * K_));

    // ---- matrix: upload + validate, hi/lo split, transpose ----
    {
        DevBuf<int> flag(1);
        PB_CUDA_CHECK(cudaMemsetAsync(flag.get(), 0, 4, st_));
        csr_upload_f64(A_, m_, n_, nnz_, rp.data(), ci.data(), val.data(), st_, flag.get());
        int h_flag = 0;
        PB_CUDA_CHECK(cudaMemcpyAsync(&h_flag, flag.get(), 4, cudaMemcpyDeviceToHost, st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        if (h_flag & 1) throw InvalidArgument("pramaan_lp: row_ptr must start at 0, be non-decreasing and end at nnz");
        if (h_flag & 2) throw InvalidArgument("pramaan_lp: col_idx entry out of bounds");
        csr_transpose(A_, AT_, st_);
    }
    auto up = [&](auto& d, const auto& h) {
        d.alloc(h.size());
        if (!h.empty())
            PB_CUDA_CHECK(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(h[0]), cudaMemcpyHostToDevice, st_));
    };
    up(cmin64_, cmin); up(rlo64_, rl); up(rhi64_, ru); up(vlo64_, vl); up(vhi64_, vu);
    up(lp_row_, lp_row); up(lp_col_, lp_col);
    if (warm) { up(xw_, xw); up(yw_, yw); }
    build_segments(rseg_, rseg);
    build_segments(cseg_, cseg);
    c_.alloc(n_); lx_.alloc(n_); ux_.alloc(n_); tau0_.alloc(n_); tau_.alloc(n_); x_.alloc(n_); xbar_.alloc(n_);
    xa_.alloc(n_); cscale_.alloc(n_);
    lr_.alloc(m_); ur_.alloc(m_); sig0_.alloc(m_); sigma_.alloc(m_); y_.alloc(m_); ya_.alloc(m_); rscale_.alloc(m_);
    ym32_.alloc(m_);
    if (!opt_.refine) { xl_.alloc(n_); yl_.alloc(m_); }
    xsum_.alloc(n_); ysum_.alloc(m_); xm64_.alloc(n_); ym64_.alloc(m_); actm64_.alloc(m_); rcm64_.alloc(n_);
    rcon_.alloc(size_t(m_) * 4); ccon_.alloc(size_t(n_) * 4);
    chunk_out_.alloc(size_t(std::max(rseg_.chunks, cseg_.chunks)) * 4 + 4);
    lp_out_.alloc(size_t(K_) * kOutWidth);
    action_.alloc(K_); inv_.alloc(K_); keep_.alloc(K_); dscale_.alloc(K_); pscale_.alloc(K_); lp_f_.alloc(K_);
    if (halpern_) {
        restart_iter_.alloc(K_);
        iter_base_.alloc(1);
        PB_CUDA_CHECK(pinned_alloc(&h_restart_iter_, sizeof(int) * K_));
        for (int q = 0; q < K_; ++q) h_restart_iter_[q] = 0;
        PB_CUDA_CHECK(cudaMemcpyAsync(restart_iter_.get(), h_restart_iter_, sizeof(int) * K_, cudaMemcpyHostToDevice, st_));
        for (int b = 0; b < 2; ++b) {
            fpr_c_[b].alloc(n_);
            fpr_r_[b].alloc(m_ > 0 ? m_ : 1);
        }
    }
    ones_.alloc(2);
    fill_kernel<<<1, 32, 0, st_>>>(ones_.get(), 2, 1.0f);
    PB_CUDA_CHECK(cudaGetLastError());
    if (m_) PB_CUDA_CHECK(cudaMemsetAsync(ysum_.get(), 0, ysum_.bytes(), st_));
    PB_CUDA_CHECK(cudaMemsetAsync(xsum_.get(), 0, xsum_.bytes(), st_));
    for (int q = 0; q < K_; ++q) h_action_[q] = kActNone;

    preconditioned_steps();          // flat operands: before pack()
    if (opt_.gather_cache >= 0) select_hot_pair(A_, AT_, dev_, st_);
    // the cluster kernel reads the flat operands (Halpern mode, unless the
    // graph path or the cooperative kernel is asked for)
    cluster_ok_ = halpern_ && (opt_.persistent == 0 || opt_.persistent == 2);
    A_.keep_flat = AT_.keep_flat = cluster_ok_;
    A_.pack(st_);
    AT_.pack(st_);
    // occupancy queries / shared-memory attributes before any graph capture
    warm_launcher<EpiDualAdapt, float, float>(dev_);
    warm_launcher<EpiPrimalAdapt, float, float>(dev_);
    warm_launcher<EpiStoreScaled, float, float>(dev_);
    warm_launcher<EpiStore<float, float>, float, float>(dev_);
    warm_launcher<EpiRowKktOut, double, float>(dev_);
    warm_launcher<EpiColKktOut, double, float>(dev_);
    warm_launcher<EpiStore<double, double>, double, double>(dev_);
    warm_launcher<EpiRowViolOut, double, double>(dev_);
    warm_launcher<EpiColResidOut, double, double>(dev_);
    estimate_step_sizes();

    // initial primal weight per LP: ||C c|| / ||R b|| on the scaled LP
    std::vector<float> hc(N), hr(M);
    PB_CUDA_CHECK(cudaMemcpyAsync(hc.data(), cscale_.get(), size_t(n_) * 4, cudaMemcpyDeviceToHost, st_));
    if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(hr.data(), rscale_.get(), size_t(m_) * 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    for (int q = 0; q < K_; ++q) {
        Lp& s = lp_[q];
        double cs = 0.0, bs = 0.0;
        for (int j = s.c0; j < s.c1; ++j) { const double v = cmin[j] * hc[j]; cs += v * v; }
        for (int i = s.r0; i < s.r1; ++i) {
            const double lo = rl[i], hi = ru[i];
            if (lo > -1e29) bs += (lo * hr[i]) * (lo * hr[i]);
            if (hi < 1e29 && !(lo > -1e29 && lo == hi)) bs += (hi * hr[i]) * (hi * hr[i]);
        }
        cs = std::sqrt(cs);
        bs = std::sqrt(bs);
        s.omega = cs > 1e-10 && bs > 1e-10 ? cs / bs : 1.0;
        if (warm) {
            const double w = warm[s.index].primal_weight;
            if (w > 0.0 && std::isfinite(w)) s.omega = w;
        }
    }
    apply_steps();
    if (halpern_) {
        set_int_kernel<<<1, 1, 0, st_>>>(iter_base_.get(), 0);
        PB_CUDA_CHECK(cudaGetLastError());
    }
    tune_products();
    if (cluster_ok_) build_cluster_lps();
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    // the packed host CSR stays for compaction
    h_rp_ = std::move(rp);
    h_ci_ = std::move(ci);
    h_val_ = std::move(val);
}

AdaptiveBatch::~AdaptiveBatch() {
    if (st_) cudaStreamSynchronize(st_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    DeviceSyncScope gate;
    if (h_action_) cudaFreeHost(h_action_);
    if (h_restart_iter_) cudaFreeHost(h_restart_iter_);
    if (h_inv_) cudaFreeHost(h_inv_);
    if (h_dscale_) cudaFreeHost(h_dscale_);
    if (h_pscale_) cudaFreeHost(h_pscale_);
    if (h_lp_f_) cudaFreeHost(h_lp_f_);
    if (h_out_) cudaFreeHost(h_out_);
    if (h_keep_) cudaFreeHost(h_keep_);
    if (h_status_) cudaFreeHost(h_status_);
    if (st_) cudaStreamDestroy(st_);
}

void AdaptiveBatch::build_segments(Segments& s, const std::vector<int>& seg_begin) {
    std::vector<int> begin, first(size_t(K_) + 1);
    for (int q = 0; q < K_; ++q) {
        first[q] = int(begin.size());
        for (int b = seg_begin[q]; b < seg_begin[q + 1]; b += kChunk) begin.push_back(b);
    }
    first[K_] = int(begin.size());
    s.chunks = int(begin.size());
    begin.push_back(seg_begin[K_]);
    // chunk c spans [begin[c], begin[c+1]) except at an LP's last chunk, which
    // ends at the LP's end; with contiguous LPs that is the next begin as well.
    s.begin.alloc(begin.size());
    s.lp_first.alloc(first.size());
    PB_CUDA_CHECK(cudaMemcpyAsync(s.begin.get(), begin.data(), begin.size() * 4, cudaMemcpyHostToDevice, st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(s.lp_first.get(), first.data(), first.size() * 4, cudaMemcpyHostToDevice, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // host vectors are freed on return
}

void AdaptiveBatch::reduce(const Segments& s, const double* contrib, int width, bool max_op, int out_off) {
    if (s.chunks > 0) {
        if (max_op)
            chunk_reduce_kernel<true><<<s.chunks, 256, 0, st_>>>(contrib, width, s.begin.get(), chunk_out_.get());
        else
            chunk_reduce_kernel<false><<<s.chunks, 256, 0, st_>>>(contrib, width, s.begin.get(), chunk_out_.get());
    }
    const int threads = K_ * width;
    if (max_op)
        lp_reduce_kernel<true><<<(threads + 255) / 256, 256, 0, st_>>>(chunk_out_.get(), width, s.lp_first.get(), K_,
                                                                      lp_out_.get(), out_off);
    else
        lp_reduce_kernel<false><<<(threads + 255) / 256, 256, 0, st_>>>(chunk_out_.get(), width, s.lp_first.get(), K_,
                                                                       lp_out_.get(), out_off);
    PB_CUDA_CHECK(cudaGetLastError());
}

void AdaptiveBatch::check_status() {
    PB_CUDA_CHECK(cudaMemcpyAsync(h_status_, status_.get(), sizeof(int), cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (*h_status_ & kDevErrTimeout) {
        PB_CUDA_CHECK(cudaMemsetAsync(status_.get(), 0, sizeof(int), st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        throw DeviceTimeout("device wait on a bulk copy exceeded its time limit; batch discarded");
    }
}

void AdaptiveBatch::fetch_out() {
    PB_CUDA_CHECK(cudaMemcpyAsync(h_out_, lp_out_.get(), sizeof(double) * K_ * kOutWidth, cudaMemcpyDeviceToHost, st_));
    check_status();   // synchronises
}

// Ruiz + Pock-Chambolle steps over the packed flat operands (row/column
// norms never mix two LPs: the packed matrix is block diagonal).
void AdaptiveBatch::preconditioned_steps() {
    DevBuf<float> r2{static_cast<size_t>(m_ > 0 ? m_ : 1)}, c2{static_cast<size_t>(n_)};
    if (m_) fill_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rscale_.get(), m_, 1.0f);
    fill_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cscale_.get(), n_, 1.0f);
    PB_CUDA_CHECK(cudaGetLastError());
    if (nnz_ > 0) {
        for (int pass = 0; pass < 10; ++pass) {
            ruiz_pass_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(A_.row_ptr.get(), A_.col.get(), A_.val.get(), m_,
                                                                cscale_.get(), rscale_.get(), r2.get());
            ruiz_pass_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(AT_.row_ptr.get(), AT_.col.get(), AT_.val.get(), n_,
                                                                rscale_.get(), cscale_.get(), c2.get());
            PB_CUDA_CHECK(cudaGetLastError());
            PB_CUDA_CHECK(cudaMemcpyAsync(rscale_.get(), r2.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
            PB_CUDA_CHECK(cudaMemcpyAsync(cscale_.get(), c2.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
        }
    }
    if (m_) pc_step_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(A_.row_ptr.get(), A_.col.get(), A_.val.get(), m_,
                                                             cscale_.get(), rscale_.get(), sig0_.get());
    pc_step_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(AT_.row_ptr.get(), AT_.col.get(), AT_.val.get(), n_,
                                                      rscale_.get(), cscale_.get(), tau0_.get());
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

// Per-LP power iteration for ||Sigma^1/2 A_k T^1/2||_2: the block-diagonal
// product runs once per step for all LPs, the Rayleigh quotient and the
// normalisation are per LP.
void AdaptiveBatch::estimate_step_sizes() {
    std::vector<double> lam(size_t(K_), 0.0);
    std::vector<char> done(size_t(K_), 0);
    for (int q = 0; q < K_; ++q) {
        const Lp& s = lp_[q];
        if (s.r1 == s.r0 || A_.nnz == 0) done[q] = 1;
        h_lp_f_[q] = float(1.0 / std::sqrt(double(s.c1 - s.c0)));
    }
    if (m_ == 0 || nnz_ == 0) {
        for (auto& s : lp_) s.eta = 0.99;
        return;
    }
    DevBuf<float> v{size_t(n_)}, t1{size_t(n_)}, u{size_t(m_)}, w{size_t(n_)}, sqrt_tau{size_t(n_)};
    PB_CUDA_CHECK(cudaMemcpyAsync(lp_f_.get(), h_lp_f_, sizeof(float) * K_, cudaMemcpyHostToDevice, st_));
    fill_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(v.get(), lp_col_.get(), lp_f_.get(), n_);
    sqrt_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(tau0_.get(), n_, sqrt_tau.get());
    PB_CUDA_CHECK(cudaGetLastError());
    for (int it = 0; it < 40; ++it) {
        mul_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(v.get(), sqrt_tau.get(), n_, t1.get());
        PB_CUDA_CHECK(cudaGetLastError());
        EpiStoreScaled e1{u.get(), sig0_.get()};
        SpmvLauncher<EpiStoreScaled, float, float, false>::launch(A_.view(false), t1.get(), e1, status_.get(), st_, dev_);
        EpiStoreScaled e2{w.get(), sqrt_tau.get()};
        SpmvLauncher<EpiStoreScaled, float, float, false>::launch(AT_.view(false), u.get(), e2, status_.get(), st_, dev_);
        dot2_contrib_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(v.get(), w.get(), n_, ccon_.get());
        PB_CUDA_CHECK(cudaGetLastError());
        reduce(cseg_, ccon_.get(), 2, false, 0);
        fetch_out();
        bool all = true;
        for (int q = 0; q < K_; ++q) {
            const double l = h_out_[size_t(q) * kOutWidth + 0];
            const double wn = std::sqrt(h_out_[size_t(q) * kOutWidth + 1]);
            float f = 1.0f;
            if (!done[q]) {
                const double prev = lam[q];
                lam[q] = l;
                if (!(wn > 0.0) || !std::isfinite(wn)) done[q] = 1;
                else {
                    f = float(1.0 / wn);
                    if (it > 5 && std::fabs(l - prev) <= 1e-4 * std::fabs(l)) done[q] = 1;
                }
            } else if (wn > 0.0 && std::isfinite(wn)) {
                f = float(1.0 / wn);
            }
            h_lp_f_[q] = f;
            all = all && done[q];
        }
        if (all) break;
        PB_CUDA_CHECK(cudaMemcpyAsync(lp_f_.get(), h_lp_f_, sizeof(float) * K_, cudaMemcpyHostToDevice, st_));
        scale_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(w.get(), lp_col_.get(), lp_f_.get(), n_, v.get());
        PB_CUDA_CHECK(cudaGetLastError());
    }
    for (int q = 0; q < K_; ++q) lp_[q].eta = 0.99 / (lam[q] > 0.0 ? std::sqrt(lam[q]) : 1.0);
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // v, w, ... are freed on return
}

// Effective steps: sigma = sigma0 * eta * omega, tau = tau0 * eta / omega; 0 for a frozen LP.
void AdaptiveBatch::apply_steps() {
    for (int q = 0; q < K_; ++q) {
        const Lp& s = lp_[q];
        h_dscale_[q] = s.active ? float(s.eta * s.omega) : 0.0f;
        h_pscale_[q] = s.active ? float(s.eta / s.omega) : 0.0f;
    }
    PB_CUDA_CHECK(cudaMemcpyAsync(dscale_.get(), h_dscale_, sizeof(float) * K_, cudaMemcpyHostToDevice, st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(pscale_.get(), h_pscale_, sizeof(float) * K_, cudaMemcpyHostToDevice, st_));
    if (m_) scale_steps_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(sig0_.get(), lp_row_.get(), dscale_.get(), m_, sigma_.get());
    scale_steps_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(tau0_.get(), lp_col_.get(), pscale_.get(), n_, tau_.get());
    PB_CUDA_CHECK(cudaGetLastError());
}

void AdaptiveBatch::iterate_once(int j, int k) {
    if (halpern_) {
        // primal first (A^T y), then the dual with the extrapolated primal (A x̄)
        double* fc = j == 0 ? fpr_c_[0].get() : (j == k - 1 ? fpr_c_[1].get() : nullptr);
        double* fr = j == 0 ? fpr_r_[0].get() : (j == k - 1 ? fpr_r_[1].get() : nullptr);
        // the anchor is the restart point, which the fold made the master: 0 in correction space
        const float* ax = nullptr;
        const float* ay = nullptr;
        // a batch of one LP reads its restart counter without per-row LP indices
        const int* lpc = K_ == 1 ? nullptr : lp_col_.get();
        const int* lpr = K_ == 1 ? nullptr : lp_row_.get();
        EpiPrimalHalpern ep{tau_.get(), c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get(), ax, lpc,
                            restart_iter_.get(), iter_base_.get(), j, fc};
        SpmvLauncher<EpiPrimalHalpern, float, float, false>::launch(AT_.view(false), y_.get(), ep, status_.get(), st_,
                                                                   dev_);
        if (m_ > 0) {
            EpiDualHalpern ed{sigma_.get(), lr_.get(), ur_.get(), ym32_.get(), y_.get(), ay, lpr,
                              restart_iter_.get(), iter_base_.get(), j, fr};
            SpmvLauncher<EpiDualHalpern, float, float, false>::launch(A_.view(false), xbar_.get(), ed, status_.get(),
                                                                     st_, dev_);
        }
        return;
    }
    if (m_ > 0) {
        EpiDualAdapt epi{sigma_.get(), lr_.get(), ur_.get(), ym32_.get(), y_.get(), ysum_.get(), ones_.get()};
        SpmvLauncher<EpiDualAdapt, float, float, false>::launch(A_.view(false), xbar_.get(), epi, status_.get(), st_, dev_);
    }
    EpiPrimalAdapt epi{tau_.get(), c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get(), xsum_.get(), ones_.get()};
    SpmvLauncher<EpiPrimalAdapt, float, float, false>::launch(AT_.view(false), y_.get(), epi, status_.get(), st_, dev_);
}

bool AdaptiveBatch::use_interval_kernel() const {
    // only on request: on the measured LPs (60 k and 12 k non-zeros) the
    // graph of dependent launches was faster per iteration (24 / 15 us) than
    // the cooperative kernel with its grid barriers (31 / 21 us)
    // (the cooperative kernel reads the operands without hot gather slots)
    return halpern_ && m_ > 0 && opt_.persistent > 0 && A_.hot == 0 && AT_.hot == 0;
}

void AdaptiveBatch::launch_interval(int k) {
    using L = SpmvSmemLayout<kSpmvWarps, kSpmvStages, false, float>;
    const bool map_a = A_.row_map.get() != nullptr, map_at = AT_.row_map.get() != nullptr;
    const int occ = interval_bps(map_a, map_at, dev_);
    const long long need = (std::max(A_.num_tiles, AT_.num_tiles) + kSpmvWarps - 1) / kSpmvWarps;
    const int grid = int(std::max<long long>(1, std::min<long long>(need, (long long)occ * device_sm_count(dev_))));
    if (gsync_.size() == 0) {
        gsync_.alloc(2);
        PB_CUDA_CHECK(cudaMemsetAsync(gsync_.get(), 0, gsync_.bytes(), st_));
    }
    const int* lpc = K_ == 1 ? nullptr : lp_col_.get();   // one LP: no per-row LP indices
    const int* lpr = K_ == 1 ? nullptr : lp_row_.get();
    EpiPrimalHalpern ep{tau_.get(), c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get(), nullptr, lpc,
                        restart_iter_.get(), iter_base_.get(), 0, nullptr};
    EpiDualHalpern ed{sigma_.get(), lr_.get(), ur_.get(), ym32_.get(), y_.get(), nullptr, lpr,
                      restart_iter_.get(), iter_base_.get(), 0, nullptr};
    const CsrView va = A_.view(false), vat = AT_.view(false);
    GridSync gs{gsync_.get(), gsync_.get() + 1, unsigned(grid)};
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(kSpmvWarps * 32);
    cfg.dynamicSmemBytes = L::bytes;
    cfg.stream = st_;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    double *c0 = fpr_c_[0].get(), *c1 = fpr_c_[1].get(), *r0 = fpr_r_[0].get(), *r1 = fpr_r_[1].get();
    const float* yp = y_.get();
    const float* xb = xbar_.get();
    int* stp = status_.get();
    if (map_a) {
        if (map_at)
            PB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, halpern_interval_kernel<true, true>, va, vat, ep, ed, yp, xb, k, c0, c1, r0, r1, gs, stp));
        else
            PB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, halpern_interval_kernel<true, false>, va, vat, ep, ed, yp, xb, k, c0, c1, r0, r1, gs, stp));
    } else {
        if (map_at)
            PB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, halpern_interval_kernel<false, true>, va, vat, ep, ed, yp, xb, k, c0, c1, r0, r1, gs, stp));
        else
            PB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, halpern_interval_kernel<false, false>, va, vat, ep, ed, yp, xb, k, c0, c1, r0, r1, gs, stp));
    }
}

// By default (persistent = 0) the cluster kernel takes the intervals once
// the layout holds few enough LPs for clusters of kClusterAutoMin blocks (the
// tail of a batch, or a single LP) and every LP has at most
// kClusterAutoMaxNnz non-zeros; persistent = 2 takes it always.  Measured on
// the rolling-horizon batch (128 LPs, T ~ U{24..336}, P ~ U{5..50}): its
// slowest LP alone (66,704 non-zeros, 300 k iterations) at 10.1 us per
// iteration against 17.9 on the tiled path; its first 16 and 32 LPs (clusters
// of 8 and 4 blocks) at 18.1 / 30.3 against 24.0 / 46.5 us, but 64 and 128
// LPs (2 blocks, 1 block) at 68.7 / 141.5 against 44.5 / 72.9 us, where the
// packed tiled products spread every LP over the whole GPU.  Clusters of 4 or
// 2 blocks taking the tail earlier did not change the 512-LP batch's time.
constexpr long long kClusterAutoMaxNnz = 1LL << 20;
// Halpern mode compacts the operand once the LPs still iterating hold less
// than this share of its non-zeros (a compaction costs ~0.1 s on the 512-LP
// batch; the frozen LPs' share of every product before it is pure waste).
constexpr double kCompactLiveShare = 0.75;
constexpr int kClusterAutoMin = 16;

void AdaptiveBatch::build_cluster_lps() {
    std::vector<int4> v;
    long long most = 0;
    for (const Lp& t : lp_) {
        if (t.r1 == t.r0 && t.c1 == t.c0) continue;   // not in the current layout
        v.push_back(make_int4(t.r0, t.r1, t.c0, t.c1));
        most = std::max(most, t.nnz);
    }
    cluster_nlps_ = int(v.size());
    cluster_auto_ = most <= kClusterAutoMaxNnz;
    cluster_lps_.alloc(v.size() > 0 ? v.size() : 1);
    if (!v.empty())
        PB_CUDA_CHECK(cudaMemcpyAsync(cluster_lps_.get(), v.data(), v.size() * sizeof(int4), cudaMemcpyHostToDevice, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // v is freed on return
    // Cluster size: the SMs shared out among the LPs (a power of two, at most
    // kClusterMax), lowered until the device can hold such a cluster.
    const int sms = device_sm_count(dev_);
    int C = 1;
    while (C * 2 <= kClusterMax && (long long)C * 2 * std::max(cluster_nlps_, 1) <= sms) C *= 2;
    static std::atomic<int> attr_set[64];
    const int slot = dev_ >= 0 && dev_ < 64 ? dev_ : 0;
    if (!attr_set[slot].exchange(1))
        PB_CUDA_CHECK(cudaFuncSetAttribute(halpern_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    for (; C > 1; C /= 2) {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(unsigned(C));
        cfg.blockDim = dim3(kClusterThreads);
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = unsigned(C);
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nc = 0;
        const cudaError_t e = cudaOccupancyMaxActiveClusters(&nc, halpern_cluster_kernel, &cfg);
        if (e == cudaSuccess && nc > 0) break;
        (void)cudaGetLastError();
    }
    cluster_size_ = C;
    cluster_auto_ = cluster_auto_ && C >= kClusterAutoMin;
    if (use_cluster_kernel()) build_cluster_long_rows(v);
}

void AdaptiveBatch::build_cluster_long_rows(const std::vector<int4>& lps) {
    std::vector<int> rp(size_t(m_) + 1, 0), cp(size_t(n_) + 1, 0);
    if (m_ > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(rp.data(), A_.row_ptr.get(), rp.size() * sizeof(int), cudaMemcpyDeviceToHost, st_));
    if (n_ > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(cp.data(), AT_.row_ptr.get(), cp.size() * sizeof(int), cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    std::vector<int4> range;
    std::vector<int> la, lat;
    for (const int4& q : lps) {
        int4 r;
        r.x = int(la.size());
        for (int i = q.x; i < q.y; ++i)
            if (rp[size_t(i) + 1] - rp[size_t(i)] > kClusterLongRow) la.push_back(i);
        r.y = int(la.size());
        r.z = int(lat.size());
        for (int j = q.z; j < q.w; ++j)
            if (cp[size_t(j) + 1] - cp[size_t(j)] > kClusterLongRow) lat.push_back(j);
        r.w = int(lat.size());
        range.push_back(r);
    }
    cluster_long_range_.alloc(range.empty() ? 1 : range.size());
    cluster_long_a_.alloc(la.empty() ? 1 : la.size());
    cluster_long_at_.alloc(lat.empty() ? 1 : lat.size());
    if (!range.empty())
        PB_CUDA_CHECK(cudaMemcpyAsync(cluster_long_range_.get(), range.data(), range.size() * sizeof(int4),
                                      cudaMemcpyHostToDevice, st_));
    if (!la.empty())
        PB_CUDA_CHECK(cudaMemcpyAsync(cluster_long_a_.get(), la.data(), la.size() * sizeof(int), cudaMemcpyHostToDevice, st_));
    if (!lat.empty())
        PB_CUDA_CHECK(cudaMemcpyAsync(cluster_long_at_.get(), lat.data(), lat.size() * sizeof(int),
                                      cudaMemcpyHostToDevice, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // the host lists are freed on return
}

bool AdaptiveBatch::use_cluster_kernel() const {
    if (!cluster_ok_ || cluster_nlps_ == 0) return false;
    return opt_.persistent == 2 || cluster_auto_;
}

void AdaptiveBatch::launch_cluster(int k) {
    const int* lpc = K_ == 1 ? nullptr : lp_col_.get();   // one LP: no per-row LP indices
    const int* lpr = K_ == 1 ? nullptr : lp_row_.get();
    EpiPrimalHalpern ep{tau_.get(), c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get(), nullptr, lpc,
                        restart_iter_.get(), iter_base_.get(), 0, nullptr};
    EpiDualHalpern ed{sigma_.get(), lr_.get(), ur_.get(), ym32_.get(), y_.get(), nullptr, lpr,
                      restart_iter_.get(), iter_base_.get(), 0, nullptr};
    const FlatCsr fa{A_.row_ptr.get(), A_.col.get(), A_.val.get()};
    const FlatCsr fat{AT_.row_ptr.get(), AT_.col.get(), AT_.val.get()};
    if (n_ > 0 && (!fat.col || !fat.val)) throw std::logic_error("cluster kernel: flat operand missing");
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(cluster_nlps_ * cluster_size_));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.stream = st_;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = unsigned(cluster_size_);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    double *c0 = fpr_c_[0].get(), *c1 = fpr_c_[1].get(), *r0 = fpr_r_[0].get(), *r1 = fpr_r_[1].get();
    const int4* lps = cluster_lps_.get();
    const float* yp = y_.get();
    const float* xb = xbar_.get();
    const int4* lr = cluster_long_range_.get();
    const int* la = cluster_long_a_.get();
    const int* lat = cluster_long_at_.get();
    if (!lr || !la || !lat) throw std::logic_error("cluster kernel: long-row lists missing");
    PB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, halpern_cluster_kernel, lps, lr, la, lat, fa, fat, ep, ed, yp, xb, k, c0,
                                     c1, r0, r1));
}

void AdaptiveBatch::iterate(int k, int iter) {
    if (k <= 0) return;
    if (halpern_) {
        set_int_kernel<<<1, 1, 0, st_>>>(iter_base_.get(), iter);
        PB_CUDA_CHECK(cudaGetLastError());
    }
    if (use_cluster_kernel()) {
        launch_cluster(k);
    } else if (use_interval_kernel()) {
        launch_interval(k);
    } else if (!opt_.use_graph || k > 4096) {
        for (int i = 0; i < k; ++i) iterate_once(i, k);
    } else {
        if (graph_iters_ != k) {
            if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
            if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
            {
                CaptureScope capture;
                PB_CUDA_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
                try {
                    for (int i = 0; i < k; ++i) iterate_once(i, k);
                } catch (...) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(st_, &g);
                    if (g) cudaGraphDestroy(g);
                    throw;
                }
                PB_CUDA_CHECK(cudaStreamEndCapture(st_, &graph_));
            }
            PB_CUDA_CHECK(cudaGraphInstantiate(&graph_exec_, graph_, 0));
            graph_iters_ = k;
        }
        PB_CUDA_CHECK(cudaGraphLaunch(graph_exec_, st_));
    }
    if (halpern_ && k == 1) {
        // the only iteration is both the first and the last one
        PB_CUDA_CHECK(cudaMemcpyAsync(fpr_c_[1].get(), fpr_c_[0].get(), size_t(n_) * 8, cudaMemcpyDeviceToDevice, st_));
        if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(fpr_r_[1].get(), fpr_r_[0].get(), size_t(m_) * 8, cudaMemcpyDeviceToDevice, st_));
    }
}

void AdaptiveBatch::materialize_average() {
    for (int q = 0; q < K_; ++q) h_inv_[q] = lp_[q].avg_count > 0 ? 1.0 / double(lp_[q].avg_count) : -1.0;
    PB_CUDA_CHECK(cudaMemcpyAsync(inv_.get(), h_inv_, sizeof(double) * K_, cudaMemcpyHostToDevice, st_));
    average_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(xsum_.get(), x_.get(), lp_col_.get(), inv_.get(), n_, xa_.get());
    if (m_) average_lp_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(ysum_.get(), y_.get(), lp_row_.get(), inv_.get(), m_, ya_.get());
    PB_CUDA_CHECK(cudaGetLastError());
}

void AdaptiveBatch::kkt(std::vector<KktSums>& cur, std::vector<KktSums>& avg, bool with_average) {
    if (with_average) materialize_average();
    const float* xs[2] = {x_.get(), xa_.get()};
    const float* ys[2] = {y_.get(), ya_.get()};
    const int candidates = with_average ? 2 : 1;
    if (m_ == 0 || !with_average) PB_CUDA_CHECK(cudaMemsetAsync(lp_out_.get(), 0, lp_out_.bytes(), st_));
    for (int k = 0; k < candidates; ++k) {
        if (m_ > 0) {
            EpiRowKktOut er{rlo64_.get(), rhi64_.get(), actm64_.get(), ym64_.get(), ys[k], rcon_.get()};
            launch_any<EpiRowKktOut, double, float>(A_, xs[k], er, status_.get(), st_, dev_);
            reduce(rseg_, rcon_.get(), 4, false, 8 * k);
        }
        EpiColKktOut ec{cmin64_.get(), vlo64_.get(), vhi64_.get(), rcm64_.get(), xm64_.get(), xs[k], ccon_.get()};
        launch_any<EpiColKktOut, double, float>(AT_, ys[k], ec, status_.get(), st_, dev_);
        reduce(cseg_, ccon_.get(), 4, false, 8 * k + 4);
    }
    fetch_out();
    cur.resize(size_t(K_));
    avg.resize(size_t(K_));
    for (int q = 0; q < K_; ++q) {
        for (int k = 0; k < 2; ++k) {
            const double* r = h_out_ + size_t(q) * kOutWidth + 8 * k;
            KktSums& o = k == 0 ? cur[q] : avg[q];
            o.pr2 = r[0] + r[4];
            o.dr2 = r[1] + r[5];
            o.dobj = r[2] + r[6];
            o.pobj = r[7];
            o.bad = r[3] > 0.0 || !std::isfinite(o.pr2) || !std::isfinite(o.dr2) || !std::isfinite(o.pobj) ||
                    !std::isfinite(o.dobj);
        }
    }
}

void AdaptiveBatch::push_actions() {
    PB_CUDA_CHECK(cudaMemcpyAsync(action_.get(), h_action_, sizeof(int) * K_, cudaMemcpyHostToDevice, st_));
}

void AdaptiveBatch::fold(bool first) {
    if (first) {
        if (xw_.size()) {
            init_master_warm_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(xw_.get(), vlo64_.get(), vhi64_.get(), n_,
                                                                       xm64_.get());
            if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(ym64_.get(), yw_.get(), ym64_.bytes(), cudaMemcpyDeviceToDevice, st_));
            xw_.reset();
            yw_.reset();
        } else {
            init_master_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(vlo64_.get(), vhi64_.get(), n_, xm64_.get());
            if (m_) PB_CUDA_CHECK(cudaMemsetAsync(ym64_.get(), 0, ym64_.bytes(), st_));
        }
        PB_CUDA_CHECK(cudaMemsetAsync(x_.get(), 0, x_.bytes(), st_));
        PB_CUDA_CHECK(cudaMemsetAsync(xbar_.get(), 0, xbar_.bytes(), st_));
        if (m_) PB_CUDA_CHECK(cudaMemsetAsync(y_.get(), 0, y_.bytes(), st_));
    } else {
        fold_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(lp_col_.get(), action_.get(), n_, xm64_.get(), x_.get(), xbar_.get());
        if (m_) fold_lp_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(lp_row_.get(), action_.get(), m_, ym64_.get(), y_.get(), nullptr);
    }
    PB_CUDA_CHECK(cudaGetLastError());
    if (m_) {
        EpiStore<double, double> e{actm64_.get()};
        launch_any<EpiStore<double, double>, double, double>(A_, xm64_.get(), e, status_.get(), st_, dev_);
        fold_rows_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rlo64_.get(), rhi64_.get(), actm64_.get(), ym64_.get(), m_,
                                                            lr_.get(), ur_.get(), ym32_.get());
        EpiStore<double, double> e2{rcm64_.get()};
        launch_any<EpiStore<double, double>, double, double>(AT_, ym64_.get(), e2, status_.get(), st_, dev_);
    } else {
        PB_CUDA_CHECK(cudaMemsetAsync(rcm64_.get(), 0, rcm64_.bytes(), st_));
    }
    fold_cols_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cmin64_.get(), vlo64_.get(), vhi64_.get(), xm64_.get(), n_,
                                                        rcm64_.get(), c_.get(), lx_.get(), ux_.get());
    PB_CUDA_CHECK(cudaGetLastError());
}

void AdaptiveBatch::solve(const pramaan_lp* lps, pramaan_solve_result* results) {
    const auto t0 = std::chrono::steady_clock::now();
    if (K_ > 0) {
        constexpr double kSufficient = 0.2, kNecessary = 0.8, kArtificial = 0.36;
        const int cf = opt_.check_frequency;
        const int max_it = opt_.max_iterations;
        const double tol = opt_.tolerance;
        const bool refine = opt_.refine != 0;
        auto converged = [&](const Lp& s, const KktSums& o, double& rp, double& rd, double& rg) {
            rp = std::sqrt(o.pr2) / (1.0 + s.b_norm);
            rd = std::sqrt(o.dr2) / (1.0 + s.c_norm);
            rg = std::fabs(o.pobj - o.dobj) / (1.0 + std::fabs(o.pobj) + std::fabs(o.dobj));
            return rp <= tol && rd <= tol && rg <= tol;
        };
        fold(true);
        if (!refine) {
            PB_CUDA_CHECK(cudaMemsetAsync(xl_.get(), 0, xl_.bytes(), st_));
            if (m_) PB_CUDA_CHECK(cudaMemsetAsync(yl_.get(), 0, yl_.bytes(), st_));
        }
        if (halpern_) {
            solve_halpern();
            const double ms =
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            finish(lps, results, ms);
            return;
        }
        std::vector<KktSums> cur, avg;
        kkt(cur, avg, true);
        for (int q = 0; q < K_; ++q) {
            Lp& s = lp_[q];
            s.kkt_restart = weighted(cur[q].pr2, cur[q].dr2, cur[q].pobj - cur[q].dobj, s.omega);
            s.kkt_prev = std::numeric_limits<double>::infinity();
            if (converged(s, cur[q], s.rel_p, s.rel_d, s.rel_gap)) {
                s.status = PRAMAAN_STATUS_OPTIMAL;
                s.active = false;
            }
        }
        apply_steps();
        int iter = 0;
        auto any_active = [&] {
            for (const Lp& s : lp_) if (s.active) return true;
            return false;
        };
        while (any_active() && iter < max_it) {
            const int chunk = std::min(cf, max_it - iter);
            iterate(chunk, iter);
            iter += chunk;
            for (Lp& s : lp_) if (s.active) s.avg_count += chunk;
            kkt(cur, avg, true);
            bool any_action = false, any_restart = false, steps_changed = false;
            for (int q = 0; q < K_; ++q) {
                Lp& s = lp_[q];
                h_action_[q] = kActNone;
                if (!s.active) continue;
                ++s.checks;
                if (cur[q].bad || avg[q].bad) {
                    s.status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
                    s.iterations = iter;
                    s.active = false;
                    steps_changed = true;
                    continue;
                }
                double rp, rd, rg;
                if (converged(s, cur[q], rp, rd, rg)) {
                    s.rel_p = rp; s.rel_d = rd; s.rel_gap = rg;
                    s.status = PRAMAAN_STATUS_OPTIMAL;
                    s.iterations = iter;
                    s.active = false;
                    steps_changed = true;
                    continue;
                }
                s.rel_p = rp; s.rel_d = rd; s.rel_gap = rg;
                double ap, ad, ag;
                if (converged(s, avg[q], ap, ad, ag)) {
                    s.rel_p = ap; s.rel_d = ad; s.rel_gap = ag;
                    s.status = PRAMAAN_STATUS_OPTIMAL;
                    s.iterations = iter;
                    s.active = false;
                    h_action_[q] = kActFreezeAverage;
                    any_action = true;
                    steps_changed = true;
                    continue;
                }
                const double kc = weighted(cur[q].pr2, cur[q].dr2, cur[q].pobj - cur[q].dobj, s.omega);
                const double ka = weighted(avg[q].pr2, avg[q].dr2, avg[q].pobj - avg[q].dobj, s.omega);
                const bool use_avg = ka < kc;
                const double kcand = use_avg ? ka : kc;
                const bool restart = kcand <= kSufficient * s.kkt_restart ||
                                     (kcand <= kNecessary * s.kkt_restart && kcand > s.kkt_prev) ||
                                     (iter - s.last_restart) >= kArtificial * iter;
                s.kkt_prev = kcand;
                if (!restart) continue;
                h_action_[q] = use_avg ? kActRestartAverage : kActRestartCurrent;
                any_action = any_restart = true;
                s.kkt_restart = kcand;
                s.kkt_prev = std::numeric_limits<double>::infinity();
                s.last_restart = iter;
                s.avg_count = 0;
                ++s.restarts;
            }
            if (any_action) {
                push_actions();
                restart_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(lp_col_.get(), action_.get(), n_, x_.get(),
                                                                     xa_.get(), xbar_.get(), xsum_.get());
                if (m_) restart_lp_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(lp_row_.get(), action_.get(), m_, y_.get(),
                                                                            ya_.get(), nullptr, ysum_.get());
                PB_CUDA_CHECK(cudaGetLastError());
            }
            if (any_restart) {
                // movement since the previous restart point in the scaled norms
                dist_contrib_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x_.get(), refine ? nullptr : xl_.get(),
                                                                       cscale_.get(), n_, ccon_.get());
                PB_CUDA_CHECK(cudaGetLastError());
                reduce(cseg_, ccon_.get(), 1, false, 0);
                if (m_) {
                    dist_contrib_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(y_.get(), refine ? nullptr : yl_.get(),
                                                                           rscale_.get(), m_, rcon_.get());
                    PB_CUDA_CHECK(cudaGetLastError());
                    reduce(rseg_, rcon_.get(), 1, false, 1);
                }
                fetch_out();
                for (int q = 0; q < K_; ++q) {
                    if (h_action_[q] != kActRestartCurrent && h_action_[q] != kActRestartAverage) continue;
                    Lp& s = lp_[q];
                    const double dx = std::sqrt(h_out_[size_t(q) * kOutWidth + 0]);
                    const double dy = m_ ? std::sqrt(h_out_[size_t(q) * kOutWidth + 1]) : 0.0;
                    if (dx > 1e-10 && dy > 1e-10) {
                        const double w = std::exp(0.5 * std::log(dy / dx) + 0.5 * std::log(s.omega));
                        if (std::isfinite(w) && w > 0.0) { s.omega = w; steps_changed = true; }
                    }
                }
                if (refine) {
                    fold(false);
                } else {
                    record_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(lp_col_.get(), action_.get(), n_, x_.get(), xl_.get());
                    if (m_) record_lp_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(lp_row_.get(), action_.get(), m_, y_.get(), yl_.get());
                    PB_CUDA_CHECK(cudaGetLastError());
                }
            }
            if (steps_changed) apply_steps();
            long long live = 0;
            for (const Lp& s : lp_) if (s.active) live += s.nnz;
            if (live > 0 && 2 * live < (long long)nnz_ && (long long)nnz_ - live >= 65536) compact();
        }
        for (Lp& s : lp_)
            if (s.status == PRAMAAN_STATUS_ITERATION_LIMIT) s.iterations = max_it;
    }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    finish(lps, results, ms);
}

// Restarted Halpern PDHG (PRAMAAN_ALGO_HALPERN): the iteration of
// EpiPrimalHalpern / EpiDualHalpern, restarts of each LP at its current
// iterate when its fixed-point residual r = ||z - T(z)|| (step-weighted)
// falls to 0.2 of its value at the last restart, or to 0.8 of it while
// growing, or after 0.36 of all iterations since that restart; termination
// on the relative KKT error of the current iterate.
void AdaptiveBatch::solve_halpern() {
    constexpr double kSufficient = 0.2, kNecessary = 0.8, kArtificial = 0.36;
    constexpr int kFrozen = INT_MIN / 4;   // restart iteration of a frozen LP: weight 1
    const int cf = opt_.check_frequency;
    const int max_it = opt_.max_iterations;
    const double tol = opt_.tolerance;
    const bool refine = opt_.refine != 0;
    auto converged = [&](const Lp& s, const KktSums& o, double& rp, double& rd, double& rg) {
        rp = std::sqrt(o.pr2) / (1.0 + s.b_norm);
        rd = std::sqrt(o.dr2) / (1.0 + s.c_norm);
        rg = std::fabs(o.pobj - o.dobj) / (1.0 + std::fabs(o.pobj) + std::fabs(o.dobj));
        return rp <= tol && rd <= tol && rg <= tol;
    };
    std::vector<KktSums> cur, avg;
    kkt(cur, avg, false);
    for (int q = 0; q < K_; ++q) {
        Lp& s = lp_[q];
        s.need_fpr0 = true;
        s.fpr_prev = std::numeric_limits<double>::infinity();
        s.last_restart = 0;
        h_restart_iter_[q] = 0;
        if (converged(s, cur[q], s.rel_p, s.rel_d, s.rel_gap)) {
            s.status = PRAMAAN_STATUS_OPTIMAL;
            s.active = false;
            h_restart_iter_[q] = kFrozen;
        }
    }
    PB_CUDA_CHECK(cudaMemcpyAsync(restart_iter_.get(), h_restart_iter_, sizeof(int) * K_, cudaMemcpyHostToDevice, st_));
    apply_steps();
    int iter = 0;
    auto any_active = [&] {
        for (const Lp& s : lp_) if (s.active) return true;
        return false;
    };
    while (any_active() && iter < max_it) {
        const int chunk = std::min(cf, max_it - iter);
        iterate(chunk, iter);
        iter += chunk;
        kkt(cur, avg, false);
        // fixed-point residual of the interval's first and last iteration (slots 8-11)
        reduce(cseg_, fpr_c_[0].get(), 1, false, 8);
        reduce(cseg_, fpr_c_[1].get(), 1, false, 10);
        if (m_) {
            reduce(rseg_, fpr_r_[0].get(), 1, false, 9);
            reduce(rseg_, fpr_r_[1].get(), 1, false, 11);
        }
        fetch_out();
        bool any_restart = false, steps_changed = false, restart_changed = false;
        for (int q = 0; q < K_; ++q) {
            Lp& s = lp_[q];
            h_action_[q] = kActNone;
            if (!s.active) continue;
            ++s.checks;
            const double* o = h_out_ + size_t(q) * kOutWidth;
            const double r_first = std::sqrt(o[8] + (m_ ? o[9] : 0.0));
            const double r_last = std::sqrt(o[10] + (m_ ? o[11] : 0.0));
            if (s.need_fpr0) {
                s.fpr0 = r_first;
                s.need_fpr0 = false;
            }
            double rp, rd, rg;
            const bool done = !cur[q].bad && converged(s, cur[q], rp, rd, rg);
            if (cur[q].bad || !std::isfinite(r_last)) {
                s.status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
            } else if (done) {
                s.status = PRAMAAN_STATUS_OPTIMAL;
            }
            if (cur[q].bad || !std::isfinite(r_last) || done) {
                if (done) { s.rel_p = rp; s.rel_d = rd; s.rel_gap = rg; }
                s.iterations = iter;
                s.active = false;
                h_restart_iter_[q] = kFrozen;
                steps_changed = restart_changed = true;
                continue;
            }
            s.rel_p = rp; s.rel_d = rd; s.rel_gap = rg;
            const bool restart = r_last <= kSufficient * s.fpr0 ||
                                 (r_last <= kNecessary * s.fpr0 && r_last > s.fpr_prev) ||
                                 (iter - s.last_restart) >= kArtificial * iter;
            s.fpr_prev = r_last;
            if (!restart) continue;
            h_action_[q] = kActRestartCurrent;
            any_restart = restart_changed = true;
            s.fpr_prev = std::numeric_limits<double>::infinity();
            s.need_fpr0 = true;
            s.last_restart = iter;
            h_restart_iter_[q] = iter;
            ++s.restarts;
        }
        if (any_restart) {
            push_actions();
            // movement since the previous restart point, in the scaled norms
            dist_contrib_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x_.get(), refine ? nullptr : xl_.get(),
                                                                   cscale_.get(), n_, ccon_.get());
            PB_CUDA_CHECK(cudaGetLastError());
            reduce(cseg_, ccon_.get(), 1, false, 0);
            if (m_) {
                dist_contrib_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(y_.get(), refine ? nullptr : yl_.get(),
                                                                       rscale_.get(), m_, rcon_.get());
                PB_CUDA_CHECK(cudaGetLastError());
                reduce(rseg_, rcon_.get(), 1, false, 1);
            }
            fetch_out();
            for (int q = 0; q < K_; ++q) {
                if (h_action_[q] != kActRestartCurrent) continue;
                Lp& s = lp_[q];
                const double dx = std::sqrt(h_out_[size_t(q) * kOutWidth + 0]);
                const double dy = m_ ? std::sqrt(h_out_[size_t(q) * kOutWidth + 1]) : 0.0;
                if (dx > 1e-10 && dy > 1e-10) {
                    const double w = std::exp(0.5 * std::log(dy / dx) + 0.5 * std::log(s.omega));
                    if (std::isfinite(w) && w > 0.0) { s.omega = w; steps_changed = true; }
                }
            }
            if (refine) {
                fold(false);   // the restart point becomes the master: the anchor is 0 again
            } else {
                record_lp_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(lp_col_.get(), action_.get(), n_, x_.get(), xl_.get());
                if (m_) record_lp_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(lp_row_.get(), action_.get(), m_, y_.get(), yl_.get());
                PB_CUDA_CHECK(cudaGetLastError());
            }
        }
        if (restart_changed)
            PB_CUDA_CHECK(cudaMemcpyAsync(restart_iter_.get(), h_restart_iter_, sizeof(int) * K_, cudaMemcpyHostToDevice, st_));
        if (steps_changed) apply_steps();
        long long live = 0;
        int live_lps = 0;
        for (const Lp& s : lp_) if (s.active) { live += s.nnz; ++live_lps; }
        // Compact when the LPs still iterating hold less than half of the
        // operand, or when so few are left that the cluster kernel would take
        // them alone (clusters of kClusterAutoMin blocks or more).
        const bool to_cluster = cluster_ok_ && opt_.persistent == 0 && !use_cluster_kernel() && live_lps > 0 &&
                                live_lps < cluster_nlps_ &&
                                (long long)live_lps * kClusterAutoMin <= device_sm_count(dev_);
        if (live > 0 && ((double(live) < kCompactLiveShare * double(nnz_) && (long long)nnz_ - live >= 65536) ||
                         to_cluster))
            compact();
    }
    for (Lp& s : lp_)
        if (s.status == PRAMAAN_STATUS_ITERATION_LIMIT) s.iterations = max_it;
}

void AdaptiveBatch::scatter_answers(const int* keep) {
    if (x_out_.size() == 0) {
        x_out_.alloc(full_n_);
        y_out_.alloc(full_m_);
    }
    const int* corig = compacted_ ? col_orig_.get() : nullptr;
    const int* rorig = compacted_ ? row_orig_.get() : nullptr;
    if (n_) scatter_answers_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(lp_col_.get(), keep, xm64_.get(), x_.get(),
                                                                     corig, n_, x_out_.get());
    if (m_) scatter_answers_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(lp_row_.get(), keep, ym64_.get(), y_.get(),
                                                                     rorig, m_, y_out_.get());
    PB_CUDA_CHECK(cudaGetLastError());
}

void AdaptiveBatch::compact() {
    // 1. answers of the LPs that leave
    for (int q = 0; q < K_; ++q) h_keep_[q] = lp_[q].active ? 1 : 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(keep_.get(), h_keep_, sizeof(int) * K_, cudaMemcpyHostToDevice, st_));
    scatter_answers(keep_.get());

    // 2. new layout: the kept LPs in their order; maps new -> current index
    std::vector<int> rmap, cmap, seg_r(static_cast<size_t>(K_) + 1), seg_c(static_cast<size_t>(K_) + 1);
    long long nz = 0;
    for (int q = 0; q < K_; ++q) {
        Lp& t = lp_[q];
        seg_r[q] = int(rmap.size());
        seg_c[q] = int(cmap.size());
        const int nr0 = int(rmap.size()), nc0 = int(cmap.size());
        if (t.active) {
            for (int i = t.r0; i < t.r1; ++i) rmap.push_back(i);
            for (int j = t.c0; j < t.c1; ++j) cmap.push_back(j);
            nz += t.nnz;
        }
        t.r0 = nr0; t.r1 = int(rmap.size());
        t.c0 = nc0; t.c1 = int(cmap.size());
    }
    seg_r[K_] = int(rmap.size());
    seg_c[K_] = int(cmap.size());
    const int nm = int(rmap.size()), nn = int(cmap.size()), nnz = int(nz);

    // 3. host CSR of the kept LPs from the original packed CSR
    std::vector<int> rp(static_cast<size_t>(nm) + 1), ci(static_cast<size_t>(nnz));
    std::vector<double> val(static_cast<size_t>(nnz));
    long long e = 0;
    for (const Lp& t : lp_) {
        if (!t.active) continue;
        for (int i = 0; i < t.or1 - t.or0; ++i) {
            rp[size_t(t.r0) + i] = int(e);
            for (int k = h_rp_[size_t(t.or0) + i]; k < h_rp_[size_t(t.or0) + i + 1]; ++k, ++e) {
                ci[size_t(e)] = h_ci_[size_t(k)] - t.oc0 + t.c0;
                val[size_t(e)] = h_val_[size_t(k)];
            }
        }
    }
    rp[size_t(nm)] = int(e);
    CsrDevice nA, nAT;
    {
        DevBuf<int> flag(1);
        PB_CUDA_CHECK(cudaMemsetAsync(flag.get(), 0, 4, st_));
        csr_upload_f64(nA, nm, nn, nnz, rp.data(), ci.data(), val.data(), st_, flag.get());
        csr_transpose(nA, nAT, st_);
        if (opt_.gather_cache >= 0) select_hot_pair(nA, nAT, dev_, st_);
        nA.keep_flat = nAT.keep_flat = cluster_ok_;
        nA.pack(st_);
        nAT.pack(st_);
    }

    // 4. the first compaction keeps the original layout for the final evaluation
    if (!compacted_) {
        full_A_ = std::move(A_);
        full_AT_ = std::move(AT_);
        copy_buf(full_cmin64_, cmin64_, st_);
        copy_buf(full_rlo64_, rlo64_, st_);
        copy_buf(full_rhi64_, rhi64_, st_);
        copy_buf(full_vlo64_, vlo64_, st_);
        copy_buf(full_vhi64_, vhi64_, st_);
        copy_buf(full_lp_row_, lp_row_, st_);
        copy_buf(full_lp_col_, lp_col_, st_);
        full_rseg_ = std::move(rseg_);
        full_cseg_ = std::move(cseg_);
    }
    A_ = std::move(nA);
    AT_ = std::move(nAT);

    // 5. every per-row / per-column array into the new layout
    DevBuf<int> dr(static_cast<size_t>(nm > 0 ? nm : 1)), dc(static_cast<size_t>(nn > 0 ? nn : 1));
    if (nm) PB_CUDA_CHECK(cudaMemcpyAsync(dr.get(), rmap.data(), size_t(nm) * 4, cudaMemcpyHostToDevice, st_));
    if (nn) PB_CUDA_CHECK(cudaMemcpyAsync(dc.get(), cmap.data(), size_t(nn) * 4, cudaMemcpyHostToDevice, st_));
    if (!compacted_) {
        copy_buf(row_orig_, dr, st_);
        copy_buf(col_orig_, dc, st_);
    } else {
        regather(row_orig_, dr, nm, st_);
        regather(col_orig_, dc, nn, st_);
    }
    for (DevBuf<double>* b : {&cmin64_, &vlo64_, &vhi64_, &xsum_, &xm64_, &rcm64_}) regather(*b, dc, nn, st_);
    for (DevBuf<float>* b : {&c_, &lx_, &ux_, &tau0_, &tau_, &x_, &xbar_, &xa_, &cscale_, &xl_})
        regather(*b, dc, nn, st_);
    regather(lp_col_, dc, nn, st_);
    for (DevBuf<double>* b : {&rlo64_, &rhi64_, &ysum_, &ym64_, &actm64_}) regather(*b, dr, nm, st_);
    for (DevBuf<float>* b : {&lr_, &ur_, &sig0_, &sigma_, &y_, &ya_, &rscale_, &ym32_, &yl_})
        regather(*b, dr, nm, st_);
    regather(lp_row_, dr, nm, st_);
    m_ = nm;
    n_ = nn;
    nnz_ = nnz;
    build_segments(rseg_, seg_r);   // synchronises: maps and host vectors may go
    build_segments(cseg_, seg_c);
    if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
    graph_iters_ = 0;
    compacted_ = true;
    ++compactions_;
    tune_products();
    if (cluster_ok_) build_cluster_lps();
}

// The launch autotuner on the current operands.  In Halpern mode it times the
// products the iteration runs (EpiPrimalHalpern / EpiDualHalpern, writing
// scratch copies of x, x̄ and y): on the rolling-horizon batches most rows
// hold two or three entries, so the epilogue's loads, which a store-only
// proxy does not have, set the best number of resident blocks.
void AdaptiveBatch::tune_products() {
    // the iteration's vectors: steps, bounds, master and correction iterates, LP indices
    mark_l2_resident(A_, AT_, 32.0 * m_ + 36.0 * n_, dev_);
    if (!halpern_) {
        autotune_operand(A_, st_, dev_, status_.get(), opt_.gather_cache, {}, 0, opt_.launch_blocks);
        autotune_operand(AT_, st_, dev_, status_.get(), opt_.gather_cache, {}, 0, opt_.launch_blocks);
        return;
    }
    DevBuf<float> xs(size_t(n_ > 0 ? n_ : 1)), xbs(size_t(n_ > 0 ? n_ : 1)), es(size_t(m_ > 0 ? m_ : 1));
    if (n_ > 0) {
        PB_CUDA_CHECK(cudaMemcpyAsync(xs.get(), x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
        PB_CUDA_CHECK(cudaMemcpyAsync(xbs.get(), xbar_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
    }
    if (m_ > 0) PB_CUDA_CHECK(cudaMemcpyAsync(es.get(), y_.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
    const int* lpc = K_ == 1 ? nullptr : lp_col_.get();
    const int* lpr = K_ == 1 ? nullptr : lp_row_.get();
    const EpiPrimalHalpern ep{tau_.get(), c_.get(), lx_.get(), ux_.get(), xs.get(), xbs.get(), nullptr, lpc,
                              restart_iter_.get(), iter_base_.get(), 0, nullptr};
    const EpiDualHalpern ed{sigma_.get(), lr_.get(), ur_.get(), ym32_.get(), es.get(), nullptr, lpr,
                            restart_iter_.get(), iter_base_.get(), 0, nullptr};
    autotune_operand(AT_, st_, dev_, status_.get(), opt_.gather_cache, [&](const CsrView& v) {
        SpmvLauncher<EpiPrimalHalpern, float, float, false>::launch(v, y_.get(), ep, status_.get(), st_, dev_);
    }, /*kind=*/3, opt_.launch_blocks);
    if (m_ > 0)
        autotune_operand(A_, st_, dev_, status_.get(), opt_.gather_cache, [&](const CsrView& v) {
            SpmvLauncher<EpiDualHalpern, float, float, false>::launch(v, xbar_.get(), ed, status_.get(), st_, dev_);
        }, /*kind=*/4, opt_.launch_blocks);
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // scratch copies are freed on return
}

void AdaptiveBatch::finish(const pramaan_lp* lps, pramaan_solve_result* results, double solve_ms) {
    std::vector<double> hx, hy, hact;
    if (K_ > 0) {
        scatter_answers(nullptr);
        // evaluation on the original layout
        const CsrDevice& A = compacted_ ? full_A_ : A_;
        const CsrDevice& AT = compacted_ ? full_AT_ : AT_;
        const DevBuf<double>& cmin = compacted_ ? full_cmin64_ : cmin64_;
        const DevBuf<double>& rlo = compacted_ ? full_rlo64_ : rlo64_;
        const DevBuf<double>& rhi = compacted_ ? full_rhi64_ : rhi64_;
        const DevBuf<double>& vlo = compacted_ ? full_vlo64_ : vlo64_;
        const DevBuf<double>& vhi = compacted_ ? full_vhi64_ : vhi64_;
        const Segments& rs = compacted_ ? full_rseg_ : rseg_;
        const Segments& cs = compacted_ ? full_cseg_ : cseg_;
        const int M = full_m_, N = full_n_;
        DevBuf<float> c32{size_t(N)}, flo{size_t(N)}, fhi{size_t(N)};
        DevBuf<double> act{size_t(M > 0 ? M : 1)};
        // the original FP32 cost (the reference criterion reads it)
        restore_cols_kernel<<<grid_1d(N), kThreads, 0, st_>>>(cmin.get(), vlo.get(), vhi.get(), N, c32.get(),
                                                               flo.get(), fhi.get());
        PB_CUDA_CHECK(cudaGetLastError());
        // reference criterion per LP (maxima): rows -> slots 0,1; columns -> slots 2,3,4
        PB_CUDA_CHECK(cudaMemsetAsync(lp_out_.get(), 0, lp_out_.bytes(), st_));
        if (M) {
            EpiStore<double, double> e{act.get()};
            launch_any<EpiStore<double, double>, double, double>(A, x_out_.get(), e, status_.get(), st_, dev_);
            EpiRowViolOut rv{rlo.get(), rhi.get(), rcon_.get()};
            launch_any<EpiRowViolOut, double, double>(A, x_out_.get(), rv, status_.get(), st_, dev_);
            reduce(rs, rcon_.get(), 2, true, 0);
        }
        EpiColResidOut cr{x_out_.get(), c32.get(), vlo.get(), vhi.get(), opt_.tolerance, ccon_.get()};
        launch_any<EpiColResidOut, double, double>(AT, y_out_.get(), cr, status_.get(), st_, dev_);
        reduce(cs, ccon_.get(), 3, true, 2);
        fetch_out();
        hx.resize(size_t(N));
        hy.resize(size_t(M));
        hact.resize(size_t(M));
        PB_CUDA_CHECK(cudaMemcpyAsync(hx.data(), x_out_.get(), size_t(N) * 8, cudaMemcpyDeviceToHost, st_));
        if (M) {
            PB_CUDA_CHECK(cudaMemcpyAsync(hy.data(), y_out_.get(), size_t(M) * 8, cudaMemcpyDeviceToHost, st_));
            PB_CUDA_CHECK(cudaMemcpyAsync(hact.data(), act.get(), size_t(M) * 8, cudaMemcpyDeviceToHost, st_));
        }
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    }
    std::vector<int> packed(size_t(count_), -1);
    for (int q = 0; q < K_; ++q) packed[lp_[q].index] = q;
    for (int k = 0; k < count_; ++k) {
        const pramaan_lp& lp = lps[k];
        pramaan_solve_result* r = &results[k];
        r->restarts = 0;
        r->checks = 0;
        r->solve_ms = solve_ms;
        r->primal_weight = 1.0;
        r->step_size = 1.0;
        r->rel_primal = r->rel_dual = r->rel_gap = std::numeric_limits<double>::quiet_NaN();
        r->compactions = compactions_;
        const int q = packed[k];
        if (q < 0) {
            // the reference's early returns (src/gpu/pdhg_solver.cu:179-192)
            r->iterations = 0;
            r->primal_residual = r->dual_residual = 0.0;
            if (lp.num_cols == 0) {
                r->status = PRAMAAN_STATUS_OPTIMAL;
                r->objective_value = lp.obj_offset;
                for (int i = 0; i < lp.num_rows; ++i) {
                    if (r->row_activity) r->row_activity[i] = 0.0;
                    if (r->y) r->y[i] = 0.0;
                }
            } else {
                r->status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
                r->objective_value = 0.0;
            }
            continue;
        }
        const Lp& s = lp_[q];
        const double* o = h_out_ + size_t(q) * kOutWidth;
        r->status = s.status;
        r->iterations = s.iterations;
        r->restarts = s.restarts;
        r->checks = s.checks;
        r->rel_primal = s.rel_p;
        r->rel_dual = s.rel_d;
        r->rel_gap = s.rel_gap;
        r->primal_weight = s.omega;
        r->step_size = s.eta;
        r->primal_residual = std::max(o[0], o[2]);
        r->dual_residual = o[3] / s.c32_inf;
        if ((o[1] > 0.0 || o[4] > 0.0) && r->status == PRAMAAN_STATUS_OPTIMAL)
            r->status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
        double obj = lp.obj_offset;
        for (int j = 0; j < lp.num_cols; ++j) {
            const double xj = hx[size_t(s.oc0) + j];
            obj += lp.obj_coeffs[j] * xj;
            if (r->x) r->x[j] = xj;
        }
        r->objective_value = obj;
        for (int i = 0; i < lp.num_rows; ++i) {
            if (r->y) r->y[i] = hy[size_t(s.or0) + i];
            if (r->row_activity) r->row_activity[i] = hact[size_t(s.or0) + i];
        }
    }
}

}  // namespace pb
