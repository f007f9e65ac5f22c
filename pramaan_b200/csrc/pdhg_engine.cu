// pdhg_engine.cu — FP32 PDHG over device-resident CSR A and stored Aᵀ.
//
// Follows the reference solve (src/gpu/pdhg_solver.cu:169-411):
//   * FP32 conversion of c (negated when maximising) and the bounds, with
//     |bound| >= 1e29 mapped to ±1e30f (:196-220);
//   * diagonal steps τ_j = 0.95/Σ_i|A_ij|, σ_i = 0.95/Σ_j|A_ij| summed in FP64
//     over the FP32 values, 0.95 when the sum is <= 1e-12 (:237-250);
//   * x₀ = clamp(0, l_x, u_x), x̄₀ = x₀, y₀ = 0 (:290-297);
//   * dual-first iteration Ax̄ → y → Aᵀy → x, x̄ (:321-337);
//   * every check_frequency iterations the FP64 residuals of
//     ComputeFp64Residuals (:107-161), optimality when both <= tolerance,
//     and the stagnation restart (:363-381);
//   * iterations = max_iterations when not optimal (:392-393); objective and
//     row activity in FP64 from the FP64 model (:402-409).
// What differs is where the work runs: the products are the merge-path
// kernels with the vector updates fused into them, the residuals are FP64
// reductions on the device (only scalars reach the host), and a check
// interval is replayed as one CUDA graph.
#include "pdhg_engine.cuh"
#include "adaptive.cuh"

#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>

namespace pb {

namespace {

constexpr int kThreads = 256;
inline int grid_1d(long long n) {
    long long g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    return int(g < 65535LL * 8 ? g : 65535LL * 8);
}

constexpr float kFltInf = 1e30f;

__global__ void prep_cost_kernel(const double* __restrict__ c64, int n, float sign,
                                 float* __restrict__ c32) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x)
        c32[j] = static_cast<float>(static_cast<double>(sign) * c64[j]);
}

__global__ void prep_bounds_kernel(const double* __restrict__ lo64, const double* __restrict__ hi64,
                                   int n, float* __restrict__ lo32, float* __restrict__ hi32) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const double lo = lo64[j], hi = hi64[j];
        lo32[j] = (lo <= -1e29) ? -kFltInf : static_cast<float>(lo);
        hi32[j] = (hi >= 1e29) ? kFltInf : static_cast<float>(hi);
    }
}

// step[i] = alpha / (float)Σ_k |(double)val[k]| over row i (sequential FP64 sum,
// row order), alpha when the sum is <= 1e-12.
__global__ void diag_step_kernel(const int* __restrict__ row_ptr, const float* __restrict__ val,
                                 int rows, float alpha, float* __restrict__ step) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < rows;
         i += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        const int b = row_ptr[i], e = row_ptr[i + 1];
        for (int k = b; k < e; ++k) s += fabs(static_cast<double>(val[k]));
        step[i] = s > 1e-12 ? alpha / static_cast<float>(s) : alpha;
    }
}

// FP32 -> FP64 copy of an iterate (the answer's x and y).
__global__ void widen_kernel(const float* __restrict__ v, int n, double* __restrict__ out) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = static_cast<double>(v[i]);
}

__global__ void init_primal_kernel(const float* __restrict__ lx, const float* __restrict__ ux,
                                   int n, float* __restrict__ x, float* __restrict__ xbar) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const float v = fmaxf(lx[j], fminf(0.0f, ux[j]));
        x[j] = v;
        xbar[j] = v;
    }
}

__global__ void copy_kernel(const float* __restrict__ src, int n, float* __restrict__ dst) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x)
        dst[j] = src[j];
}

template <typename T>
void upload(DevBuf<T>& d, const T* h, size_t n, cudaStream_t st) {
    d.alloc(n);
    if (n) PB_CUDA_CHECK(cudaMemcpyAsync(d.get(), h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}

}  // namespace

void validate_lp(const pramaan_lp& lp) {
    if (lp.num_rows < 0 || lp.num_cols < 0 || lp.nnz < 0)
        throw InvalidArgument("pramaan_lp: negative dimension");
    if (lp.num_cols > 0 && (!lp.obj_coeffs || !lp.var_lower || !lp.var_upper))
        throw InvalidArgument("pramaan_lp: missing column arrays");
    if (lp.num_rows > 0 && (!lp.row_lower || !lp.row_upper || !lp.row_ptr))
        throw InvalidArgument("pramaan_lp: missing row arrays");
    if (lp.nnz > 0 && (!lp.col_idx || !lp.values))
        throw InvalidArgument("pramaan_lp: missing non-zero arrays");
    if (lp.obj_sense != PRAMAAN_MINIMIZE && lp.obj_sense != PRAMAAN_MAXIMIZE)
        throw InvalidArgument("pramaan_lp: obj_sense must be PRAMAAN_MINIMIZE or PRAMAAN_MAXIMIZE");
}

void validate_options(const pramaan_pdhg_options& opt) {
    if (opt.check_frequency < 1) throw InvalidArgument("pdhg options: check_frequency must be >= 1");
    if (opt.max_iterations < 0) throw InvalidArgument("pdhg options: max_iterations must be >= 0");
    if (!(opt.tolerance >= 0.0)) throw InvalidArgument("pdhg options: tolerance must be >= 0");
    if (opt.algorithm != PRAMAAN_ALGO_REFERENCE && opt.algorithm != PRAMAAN_ALGO_ADAPTIVE &&
        opt.algorithm != PRAMAAN_ALGO_HALPERN)
        throw InvalidArgument("pdhg options: unknown algorithm");
    if (opt.termination != PRAMAAN_TERM_REFERENCE && opt.termination != PRAMAAN_TERM_RELATIVE_KKT)
        throw InvalidArgument("pdhg options: unknown termination criterion");
    if (opt.algorithm == PRAMAAN_ALGO_REFERENCE && opt.termination != PRAMAAN_TERM_REFERENCE)
        throw InvalidArgument("pdhg options: the reference algorithm uses the reference criterion");
    if (opt.algorithm != PRAMAAN_ALGO_REFERENCE && opt.termination != PRAMAAN_TERM_RELATIVE_KKT)
        throw InvalidArgument("pdhg options: the adaptive and Halpern algorithms terminate on the relative KKT "
                              "error (PRAMAAN_TERM_RELATIVE_KKT)");
    if (opt.refine != 0 && opt.refine != 1) throw InvalidArgument("pdhg options: refine must be 0 or 1");
    if (opt.persistent < -1 || opt.persistent > 2) throw InvalidArgument("pdhg options: persistent must be -1, 0, 1 or 2");
    if (opt.gather_cache < -1 || opt.gather_cache > 1) throw InvalidArgument("pdhg options: gather_cache must be -1, 0 or 1");
    if (opt.launch_blocks < 0 || opt.launch_blocks > 64) throw InvalidArgument("pdhg options: launch_blocks must be 0..64");
    if (opt.panel_split < -1 || opt.panel_split > 1000000)
        throw InvalidArgument("pdhg options: panel_split must be -1, 0, 1 or a row length up to 1000000");
    if (opt.algorithm == PRAMAAN_ALGO_HALPERN && opt.refine != 1)
        throw InvalidArgument("pdhg options: the Halpern algorithm runs on FP64 master iterates (refine = 1)");
}

PdhgEngine::PdhgEngine(const pramaan_lp& lp, const pramaan_pdhg_options& opt) : opt_(opt) {
    validate_lp(lp);
    validate_options(opt);
    dev_ = opt.device;
    m_ = lp.num_rows;
    n_ = lp.num_cols;
    PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    PB_CUDA_CHECK(pinned_alloc(&h_slots_, sizeof(double) * kSlotCount));
    PB_CUDA_CHECK(pinned_alloc(&h_status_, sizeof(int)));
    status_.alloc(1);
    slots_.alloc(kSlotCount);
    PB_CUDA_CHECK(cudaMemsetAsync(status_.get(), 0, sizeof(int), st_));

    // ---- matrix: upload + validate, FP32 hi/lo split, stored transpose ----
    {
        DevBuf<int> flag(1);
        PB_CUDA_CHECK(cudaMemsetAsync(flag.get(), 0, 4, st_));
        static const int zero_rp = 0;
        csr_upload_f64(A_, m_, n_, lp.nnz, m_ > 0 ? lp.row_ptr : &zero_rp, lp.col_idx, lp.values,
                       st_, flag.get());
        int h_flag = 0;
        PB_CUDA_CHECK(cudaMemcpyAsync(&h_flag, flag.get(), 4, cudaMemcpyDeviceToHost, st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        if (h_flag & 1) throw InvalidArgument("pramaan_lp: row_ptr must start at 0, be non-decreasing and end at nnz");
        if (h_flag & 2) throw InvalidArgument("pramaan_lp: col_idx entry out of bounds");
        csr_transpose(A_, AT_, st_);
    }

    // ---- vectors ----
    const float obj_sign = lp.obj_sense == PRAMAAN_MAXIMIZE ? -1.0f : 1.0f;
    {
        double cn = 1.0;
        for (int j = 0; j < n_; ++j) {
            const float cj = static_cast<float>(static_cast<double>(obj_sign) * lp.obj_coeffs[j]);
            cn = std::max(cn, static_cast<double>(std::fabs(cj)));
        }
        c_norm_ = cn;
    }
    DevBuf<double> c64;
    upload(c64, lp.obj_coeffs, size_t(n_), st_);
    upload(vlo64_, lp.var_lower, size_t(n_), st_);
    upload(vhi64_, lp.var_upper, size_t(n_), st_);
    upload(rlo64_, lp.row_lower, size_t(m_), st_);
    upload(rhi64_, lp.row_upper, size_t(m_), st_);
    c_.alloc(n_); lx_.alloc(n_); ux_.alloc(n_); tau_.alloc(n_); x_.alloc(n_); xbar_.alloc(n_);
    lr_.alloc(m_); ur_.alloc(m_); sigma_.alloc(m_); y_.alloc(m_);
    if (n_ > 0) {
        prep_cost_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(c64.get(), n_, obj_sign, c_.get());
        prep_bounds_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(vlo64_.get(), vhi64_.get(), n_,
                                                               lx_.get(), ux_.get());
        diag_step_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(AT_.row_ptr.get(), AT_.val.get(), n_,
                                                             0.95f, tau_.get());
        init_primal_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(lx_.get(), ux_.get(), n_, x_.get(),
                                                              xbar_.get());
        PB_CUDA_CHECK(cudaGetLastError());
    }
    if (m_ > 0) {
        prep_bounds_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rlo64_.get(), rhi64_.get(), m_,
                                                               lr_.get(), ur_.get());
        diag_step_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(A_.row_ptr.get(), A_.val.get(), m_,
                                                             0.95f, sigma_.get());
        PB_CUDA_CHECK(cudaGetLastError());
        PB_CUDA_CHECK(cudaMemsetAsync(y_.get(), 0, size_t(m_) * 4, st_));
    }
    // Adaptive mode: Ruiz + Pock-Chambolle steps replace the reference steps
    // (they also read the flat operands).
    if (opt.algorithm == PRAMAAN_ALGO_ADAPTIVE) setup_adaptive(lp);
    // The step sizes above read the flat operands; interleave them into tile records now.
    if (opt.gather_cache >= 0) select_hot_pair(A_, AT_, dev_, st_);
    // Reference mode: the long rows of a power-law A go to the column-panel
    // product (built from the flat operand, so before pack()).
    if (!adaptive_) {
        build_panel_split(A_, panel_, opt.panel_split, dev_, st_);
        build_panel_hot(A_, AT_, panel_, panel_t_, opt.gather_cache, dev_, st_);
    }
    A_.pack(st_);
    AT_.pack(st_);
    // the iteration's vectors: sigma, bounds, y (rows); tau, c, bounds, x, x̄ (columns), plus the gathers
    mark_l2_resident(A_, AT_, 20.0 * m_ + 28.0 * n_, dev_);
    // Occupancy queries / smem attributes before any graph capture.
    SpmvLauncher<EpiDualRef, float, float, false>::blocks_per_sm(dev_);
    SpmvLauncher<EpiPrimalRef, float, float, false>::blocks_per_sm(dev_);
    SpmvLauncher<EpiRowViolRef, double, float, true>::blocks_per_sm(dev_);
    SpmvLauncher<EpiRowViolRef, double, float, false>::blocks_per_sm(dev_);
    SpmvLauncher<EpiColResidRef, double, float, false>::blocks_per_sm(dev_);
    SpmvLauncher<EpiStore<double, double>, double, float, true>::blocks_per_sm(dev_);
    SpmvLauncher<EpiStore<double, double>, double, float, false>::blocks_per_sm(dev_);
    SpmvLauncher<EpiStore<float, float>, float, float, false>::blocks_per_sm(dev_);
    SpmvLauncher<EpiPrimalRefAdd, float, float, false>::blocks_per_sm(dev_);
    if (panel_.active) panel_prepare(dev_);
    if (!adaptive_) {
        // The tuner times the fused products of the reference iteration
        // themselves, writing scratch copies of y, x and x̄.
        DevBuf<float> ys(size_t(m_ > 0 ? m_ : 1)), xs(size_t(n_ > 0 ? n_ : 1)), xbs(size_t(n_ > 0 ? n_ : 1));
        if (m_ > 0) PB_CUDA_CHECK(cudaMemcpyAsync(ys.get(), y_.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
        if (n_ > 0) {
            PB_CUDA_CHECK(cudaMemcpyAsync(xs.get(), x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
            PB_CUDA_CHECK(cudaMemcpyAsync(xbs.get(), xbar_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
        }
        const EpiDualRef de{sigma_.get(), lr_.get(), ur_.get(), ys.get()};
        const EpiPrimalRef pe{tau_.get(), c_.get(), lx_.get(), ux_.get(), xs.get(), xbs.get()};
        // With the panel split the tiled dual product covers the short rows only.
        autotune_operand(panel_.active ? panel_.S : A_, st_, dev_, status_.get(), opt.gather_cache,
                         [&](const CsrView& v) {
            SpmvLauncher<EpiDualRef, float, float, false>::launch(v, xbar_.get(), de, status_.get(), st_, dev_);
        }, /*kind=*/1, opt.launch_blocks);
        if (panel_t_.active) {
            // the tiled primal product covers the entries outside the hot rows
            const EpiPrimalRefAdd pa{pe, panel_t_.part.get()};
            autotune_operand(panel_t_.rest, st_, dev_, status_.get(), opt.gather_cache, [&](const CsrView& v) {
                SpmvLauncher<EpiPrimalRefAdd, float, float, false>::launch(v, y_.get(), pa, status_.get(), st_, dev_);
            }, /*kind=*/5, opt.launch_blocks);
        } else {
            autotune_operand(AT_, st_, dev_, status_.get(), opt.gather_cache, [&](const CsrView& v) {
                SpmvLauncher<EpiPrimalRef, float, float, false>::launch(v, y_.get(), pe, status_.get(), st_, dev_);
            }, /*kind=*/2, opt.launch_blocks);
        }
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // scratch copies are freed on return
    } else {
        // The FP32 product kernels share one shared-memory layout, so the grid the
        // tuner picks for the store-only kernel carries over to the adaptive epilogues.
        autotune_operand(A_, st_, dev_, status_.get(), opt.gather_cache, {}, 0, opt.launch_blocks);
        autotune_operand(AT_, st_, dev_, status_.get(), opt.gather_cache, {}, 0, opt.launch_blocks);
    }
    if (adaptive_) {
        SpmvLauncher<EpiDualAdapt, float, float, false>::blocks_per_sm(dev_);
        SpmvLauncher<EpiPrimalAdapt, float, float, false>::blocks_per_sm(dev_);
        SpmvLauncher<EpiStoreScaled, float, float, false>::blocks_per_sm(dev_);
        SpmvLauncher<EpiRowKkt, double, float, true>::blocks_per_sm(dev_);
        SpmvLauncher<EpiRowKkt, double, float, false>::blocks_per_sm(dev_);
        SpmvLauncher<EpiColKkt, double, float, true>::blocks_per_sm(dev_);
        SpmvLauncher<EpiColKkt, double, float, false>::blocks_per_sm(dev_);
        SpmvLauncher<EpiStore<double, double>, double, double, true>::blocks_per_sm(dev_);
        SpmvLauncher<EpiStore<double, double>, double, double, false>::blocks_per_sm(dev_);
        eta_ = 0.99 / estimate_operator_norm();
        // initial primal weight ||C c|| / ||R b|| on the scaled problem
        std::vector<float> hc(static_cast<size_t>(n_)), hr(static_cast<size_t>(m_));
        if (n_) PB_CUDA_CHECK(cudaMemcpyAsync(hc.data(), cscale_.get(), size_t(n_) * 4, cudaMemcpyDeviceToHost, st_));
        if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(hr.data(), rscale_.get(), size_t(m_) * 4, cudaMemcpyDeviceToHost, st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        const double sgn = lp.obj_sense == PRAMAAN_MAXIMIZE ? -1.0 : 1.0;
        double cs = 0.0, bs = 0.0;
        for (int j = 0; j < n_; ++j) { const double v = sgn * lp.obj_coeffs[j] * hc[j]; cs += v * v; }
        for (int i = 0; i < m_; ++i) {
            const double lo = lp.row_lower[i], hi = lp.row_upper[i];
            if (lo > -1e29) bs += (lo * hr[i]) * (lo * hr[i]);
            if (hi < 1e29 && !(lo > -1e29 && lo == hi)) bs += (hi * hr[i]) * (hi * hr[i]);
        }
        cs = std::sqrt(cs);
        bs = std::sqrt(bs);
        set_weight(cs > 1e-10 && bs > 1e-10 ? cs / bs : 1.0);
    }
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));   // c64 is freed on return
}

PdhgEngine::~PdhgEngine() {
    if (st_) cudaStreamSynchronize(st_);
    if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
    if (graph_) cudaGraphDestroy(graph_);
    for (auto& e : ev_pool_) { cudaEventDestroy(e.a); cudaEventDestroy(e.b); }
    {
        DeviceSyncScope gate;
        if (h_slots_) cudaFreeHost(h_slots_);
        if (h_status_) cudaFreeHost(h_status_);
        if (h_red_) cudaFreeHost(h_red_);
    }
    if (st_) cudaStreamDestroy(st_);
}

void PdhgEngine::launch_dual() {
    if (m_ <= 0) return;
    if (adaptive_) {
        EpiDualAdapt epi{sigma_.get(), lr_.get(), ur_.get(), ym32_.get(), y_.get(), ysum_.get(), scal_.get()};
        SpmvLauncher<EpiDualAdapt, float, float, false>::launch(A_.view(false), xbar_.get(), epi,
                                                                status_.get(), st_, dev_);
        return;
    }
    EpiDualRef epi{sigma_.get(), lr_.get(), ur_.get(), y_.get()};
    if (panel_.active) {
        panel_launch(panel_, n_, xbar_.get(), epi, status_.get(), st_, dev_);
        return;
    }
    SpmvLauncher<EpiDualRef, float, float, false>::launch(A_.view(false), xbar_.get(), epi,
                                                          status_.get(), st_, dev_);
}

void PdhgEngine::launch_primal() {
    if (n_ <= 0) return;
    if (adaptive_) {
        EpiPrimalAdapt epi{tau_.get(), c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get(),
                           xsum_.get(), scal_.get()};
        SpmvLauncher<EpiPrimalAdapt, float, float, false>::launch(AT_.view(false), y_.get(), epi,
                                                                  status_.get(), st_, dev_);
        return;
    }
    EpiPrimalRef epi{tau_.get(), c_.get(), lx_.get(), ux_.get(), x_.get(), xbar_.get()};
    if (panel_t_.active) {
        // the hot rows' part per column (panel kernel), then the other entries
        // with the primal update adding that part
        panel_product_launch(panel_t_.view(n_), y_.get(), status_.get(), st_);
        const EpiPrimalRefAdd pa{epi, panel_t_.part.get()};
        SpmvLauncher<EpiPrimalRefAdd, float, float, false>::launch(panel_t_.rest.view(false), y_.get(), pa,
                                                                   status_.get(), st_, dev_);
        return;
    }
    SpmvLauncher<EpiPrimalRef, float, float, false>::launch(AT_.view(false), y_.get(), epi,
                                                            status_.get(), st_, dev_);
}

void PdhgEngine::iterate_once() {
    if (!opt_.profile_kernels) {
        launch_dual();
        launch_primal();
        return;
    }
    auto timed = [&](int kind, auto&& fn) {
        if (ev_used_ == ev_pool_.size()) {
            if (ev_pool_.size() >= 4096) drain_events();
            if (ev_used_ == ev_pool_.size()) {
                EvPair p;
                PB_CUDA_CHECK(cudaEventCreate(&p.a));
                PB_CUDA_CHECK(cudaEventCreate(&p.b));
                ev_pool_.push_back(p);
            }
        }
        EvPair& p = ev_pool_[ev_used_++];
        p.kind = kind;
        PB_CUDA_CHECK(cudaEventRecord(p.a, st_));
        fn();
        PB_CUDA_CHECK(cudaEventRecord(p.b, st_));
    };
    if (m_ > 0) timed(0, [&] { launch_dual(); });
    if (n_ > 0) timed(1, [&] { launch_primal(); });
}

void PdhgEngine::drain_events() {
    if (ev_used_ == 0) return;
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    for (size_t i = 0; i < ev_used_; ++i) {
        float ms = 0.f;
        PB_CUDA_CHECK(cudaEventElapsedTime(&ms, ev_pool_[i].a, ev_pool_[i].b));
        if (ev_pool_[i].kind == 0) ms_dual_ += ms; else ms_primal_ += ms;
        // kernels of one product: the main kernel and, when rows cross tiles, their completion
        // (with the panel split: the panel kernel, the short rows' product, the finish kernel)
        launches_ += ev_pool_[i].kind == 0
                         ? (panel_.active ? panel_launches<EpiDualRef>(panel_)
                                          : SpmvLauncher<EpiDualRef, float, float, false>::launches(A_.view(false)))
                         : (panel_t_.active
                                ? 1 + SpmvLauncher<EpiPrimalRefAdd, float, float, false>::launches(panel_t_.rest.view(false))
                                : SpmvLauncher<EpiPrimalRef, float, float, false>::launches(AT_.view(false)));
    }
    ev_used_ = 0;
}

void PdhgEngine::kernel_times(double* ms_dual, double* ms_primal, long long* launches, bool reset) {
    drain_events();
    if (ms_dual) *ms_dual = ms_dual_;
    if (ms_primal) *ms_primal = ms_primal_;
    if (launches) *launches = launches_;
    if (reset) { ms_dual_ = ms_primal_ = 0.0; launches_ = 0; }
}

double PdhgEngine::bytes_dual() const {
    // SpMV bytes + σ, l_r, u_r, y read + y written.
    return m_ > 0 ? A_.spmv_bytes() - 4.0 * m_ + 20.0 * m_ : 0.0;
}

double PdhgEngine::bytes_primal() const {
    // SpMV bytes + τ, c, l_x, u_x, x read + x, x̄ written.
    return n_ > 0 ? AT_.spmv_bytes() - 4.0 * n_ + 28.0 * n_ : 0.0;
}

void PdhgEngine::build_graph(int k) {
    if (graph_exec_) { cudaGraphExecDestroy(graph_exec_); graph_exec_ = nullptr; }
    if (graph_) { cudaGraphDestroy(graph_); graph_ = nullptr; }
    {
        CaptureScope capture;
        PB_CUDA_CHECK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
        try {
            for (int i = 0; i < k; ++i) iterate_once();
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

void PdhgEngine::iterate(int k) {
    if (k <= 0) return;
    const bool graph = opt_.use_graph && !opt_.profile_kernels && k <= 4096;
    if (graph) {
        if (graph_iters_ != k) build_graph(k);
        PB_CUDA_CHECK(cudaGraphLaunch(graph_exec_, st_));
    } else {
        for (int i = 0; i < k; ++i) iterate_once();
    }
}

void PdhgEngine::synchronize() {
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    check_device_status();
}

void PdhgEngine::check_device_status() {
    PB_CUDA_CHECK(cudaMemcpyAsync(h_status_, status_.get(), sizeof(int), cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (*h_status_ & kDevErrTimeout) {
        PB_CUDA_CHECK(cudaMemsetAsync(status_.get(), 0, sizeof(int), st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        throw DeviceTimeout("device wait on a bulk copy exceeded its time limit; iterate discarded");
    }
}

void PdhgEngine::residuals(double& pv, double& dv, bool& nonfinite) {
    PB_CUDA_CHECK(cudaMemsetAsync(slots_.get(), 0, sizeof(double) * kSlotCount, st_));
    if (m_ > 0) {
        EpiRowViolRef epi{rlo64_.get(), rhi64_.get(), slots_.get()};
        if (A_.has_lo)
            SpmvLauncher<EpiRowViolRef, double, float, true>::launch(A_.view(true), x_.get(), epi,
                                                                     status_.get(), st_, dev_);
        else
            SpmvLauncher<EpiRowViolRef, double, float, false>::launch(A_.view(false), x_.get(), epi,
                                                                      status_.get(), st_, dev_);
    }
    if (n_ > 0) {
        EpiColResidRef epi{x_.get(), c_.get(), vlo64_.get(), vhi64_.get(), opt_.tolerance, slots_.get()};
        SpmvLauncher<EpiColResidRef, double, float, false>::launch(AT_.view(false), y_.get(), epi,
                                                                   status_.get(), st_, dev_);
    }
    PB_CUDA_CHECK(cudaMemcpyAsync(h_slots_, slots_.get(), sizeof(double) * kSlotCount,
                                  cudaMemcpyDeviceToHost, st_));
    check_device_status();   // synchronises
    pv = std::max(h_slots_[kSlotRowViol], h_slots_[kSlotBoundViol]);
    dv = h_slots_[kSlotDualViol] / c_norm_;
    nonfinite = h_slots_[kSlotNonFinite] > 0.0;
}

void PdhgEngine::restart() {
    if (m_ > 0) PB_CUDA_CHECK(cudaMemsetAsync(y_.get(), 0, size_t(m_) * 4, st_));
    if (n_ > 0) {
        copy_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x_.get(), n_, xbar_.get());
        PB_CUDA_CHECK(cudaGetLastError());
    }
}

void PdhgEngine::get_iterates(float* h_x, float* h_y) {
    if (h_x && n_ > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(h_x, x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToHost, st_));
    if (h_y && m_ > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(h_y, y_.get(), size_t(m_) * 4, cudaMemcpyDeviceToHost, st_));
    synchronize();
}

void PdhgEngine::solve(const pramaan_lp& lp, pramaan_solve_result* res) {
    res->status = PRAMAAN_STATUS_ITERATION_LIMIT;
    res->iterations = 0;
    res->restarts = 0;
    res->checks = 0;
    res->rel_primal = res->rel_dual = res->rel_gap = std::numeric_limits<double>::quiet_NaN();
    res->primal_weight = 1.0;
    res->step_size = 1.0;

    const int max_it = opt_.max_iterations;
    const int cf = opt_.check_frequency;
    const double tol = opt_.tolerance;
    double best = std::numeric_limits<double>::infinity();
    int stagnation = 0, restarts = 0;
    constexpr int kRestartPeriod = 8;   // checks without a 1% improvement
    constexpr int kMaxRestarts = 10;
    bool numerical_failure = false;

    int iter = adaptive_ ? max_it : 0;   // the adaptive loop lives in solve_adaptive
    if (adaptive_) {
        solve_adaptive(res);
        restarts = res->restarts;
        numerical_failure = res->status == PRAMAAN_STATUS_NUMERICAL_FAILURE;
    }
    while (iter < max_it) {
        const int chunk = std::min(cf - (iter % cf), max_it - iter);
        iterate(chunk);
        iter += chunk;
        if (iter % cf != 0) continue;
        double pv = 0, dv = 0;
        bool nonfinite = false;
        residuals(pv, dv, nonfinite);
        ++res->checks;
        res->primal_residual = pv;
        res->dual_residual = dv;
        if (nonfinite) { numerical_failure = true; res->iterations = iter; break; }
        if (pv <= tol && dv <= tol) {
            res->status = PRAMAAN_STATUS_OPTIMAL;
            res->iterations = iter;
            break;
        }
        const double combined = pv + dv;
        if (combined > tol * 10.0) {
            if (combined < best * 0.99) { best = combined; stagnation = 0; }
            else ++stagnation;
            if (stagnation >= kRestartPeriod && restarts < kMaxRestarts) {
                restart();
                stagnation = 0;
                best = std::numeric_limits<double>::infinity();
                ++restarts;
            }
        }
    }
    res->restarts = restarts;
    if (numerical_failure) res->status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
    if (res->status == PRAMAAN_STATUS_ITERATION_LIMIT) res->iterations = max_it;

    // ---- final residuals, x, y, objective, row activity ----
    {
        double pv = 0, dv = 0;
        bool nonfinite = false;
        if (master_out_) reference_residuals64(pv, dv, nonfinite);
        else residuals(pv, dv, nonfinite);
        res->primal_residual = pv;
        res->dual_residual = dv;
        if (nonfinite && res->status == PRAMAAN_STATUS_OPTIMAL)
            res->status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
    }
    // x and y in FP64 straight into the caller's arrays (x into a host copy
    // when the caller passed none, for the objective); FP32 iterates are
    // widened on the device, so one copy crosses PCIe
    std::vector<double> hx_own;
    double* hx = res->x;
    if (!hx && n_ > 0) {
        hx_own.resize(static_cast<size_t>(n_));
        hx = hx_own.data();
    }
    double* hy = m_ > 0 ? res->y : nullptr;
    if (master_out_) {
        // the FP64 master iterate is the answer
        if (n_) PB_CUDA_CHECK(cudaMemcpyAsync(hx, x64_.get(), size_t(n_) * 8, cudaMemcpyDeviceToHost, st_));
        if (hy) PB_CUDA_CHECK(cudaMemcpyAsync(hy, y64_.get(), size_t(m_) * 8, cudaMemcpyDeviceToHost, st_));
        synchronize();
    } else {
        DevBuf<double> xd(static_cast<size_t>(n_)), yd(static_cast<size_t>(hy ? m_ : 0));
        if (n_) {
            widen_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x_.get(), n_, xd.get());
            PB_CUDA_CHECK(cudaGetLastError());
            PB_CUDA_CHECK(cudaMemcpyAsync(hx, xd.get(), size_t(n_) * 8, cudaMemcpyDeviceToHost, st_));
        }
        if (hy) {
            widen_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(y_.get(), m_, yd.get());
            PB_CUDA_CHECK(cudaGetLastError());
            PB_CUDA_CHECK(cudaMemcpyAsync(hy, yd.get(), size_t(m_) * 8, cudaMemcpyDeviceToHost, st_));
        }
        synchronize();
    }
    double obj = lp.obj_offset;
    for (int j = 0; j < n_; ++j) obj += lp.obj_coeffs[j] * hx[j];
    res->objective_value = obj;
    if (res->row_activity && m_ > 0) {
        DevBuf<double> act{size_t(m_)};
        EpiStore<double, double> epi{act.get()};
        if (master_out_) {
            if (A_.has_lo)
                SpmvLauncher<EpiStore<double, double>, double, double, true>::launch(
                    A_.view(true), x64_.get(), epi, status_.get(), st_, dev_);
            else
                SpmvLauncher<EpiStore<double, double>, double, double, false>::launch(
                    A_.view(false), x64_.get(), epi, status_.get(), st_, dev_);
        } else if (A_.has_lo) {
            SpmvLauncher<EpiStore<double, double>, double, float, true>::launch(
                A_.view(true), x_.get(), epi, status_.get(), st_, dev_);
        } else {
            SpmvLauncher<EpiStore<double, double>, double, float, false>::launch(
                A_.view(false), x_.get(), epi, status_.get(), st_, dev_);
        }
        PB_CUDA_CHECK(cudaMemcpyAsync(res->row_activity, act.get(), size_t(m_) * 8,
                                      cudaMemcpyDeviceToHost, st_));
        synchronize();
    }
}

// Reference criterion (src/gpu/pdhg_solver.cu:107-161) evaluated on the FP64
// master iterate of a refined solve.
void PdhgEngine::reference_residuals64(double& pv, double& dv, bool& nonfinite) {
    PB_CUDA_CHECK(cudaMemsetAsync(slots_.get(), 0, sizeof(double) * kSlotCount, st_));
    if (m_ > 0) {
        EpiRowViolRef epi{rlo64_.get(), rhi64_.get(), slots_.get()};
        if (A_.has_lo)
            SpmvLauncher<EpiRowViolRef, double, double, true>::launch(A_.view(true), x64_.get(), epi,
                                                                      status_.get(), st_, dev_);
        else
            SpmvLauncher<EpiRowViolRef, double, double, false>::launch(A_.view(false), x64_.get(), epi,
                                                                       status_.get(), st_, dev_);
    }
    if (n_ > 0) {
        EpiColResidRefT<double> epi{x64_.get(), c_.get(), vlo64_.get(), vhi64_.get(), opt_.tolerance,
                                    slots_.get()};
        SpmvLauncher<EpiColResidRefT<double>, double, double, false>::launch(AT_.view(false), y64_.get(), epi,
                                                                             status_.get(), st_, dev_);
    }
    PB_CUDA_CHECK(cudaMemcpyAsync(h_slots_, slots_.get(), sizeof(double) * kSlotCount,
                                  cudaMemcpyDeviceToHost, st_));
    check_device_status();
    pv = std::max(h_slots_[kSlotRowViol], h_slots_[kSlotBoundViol]);
    dv = h_slots_[kSlotDualViol] / c_norm_;
    nonfinite = h_slots_[kSlotNonFinite] > 0.0;
}

}  // namespace pb
