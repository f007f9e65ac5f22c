// pdhg_adaptive.cu — the adaptive restarted PDHG mode (PRAMAAN_ALGO_ADAPTIVE).
//
// Same per-element iteration as the reference (dual-first: A x̄ -> y, A^T y ->
// x, x̄), with the extensions of PDLP (Applegate et al., "Practical large-scale
// linear programming using primal-dual hybrid gradient", NeurIPS 2021) and
// cuPDLP.jl (Lu & Yang, 2023), restated here from their published
// descriptions:
//   * preconditioning: 10 Ruiz passes (row/column inf-norm equilibration,
//     scales R, C) then Pock-Chambolle with alpha = 1 on the scaled matrix,
//     giving sigma'_i = 1/sum_j |R_i a_ij C_j| and tau'_j = 1/sum_i |...|;
//     in the original variables the steps are sigma_i = R_i^2 sigma'_i and
//     tau_j = C_j^2 tau'_j, so the matrix itself is never rewritten;
//   * step size eta = 0.99 / ||Sigma^1/2 A T^1/2||_2 (power iteration) and
//     primal weight omega (initially ||C c|| / ||R b||), applied as the
//     device scalars eta/omega (primal) and eta*omega (dual);
//   * the averaged iterate (uniform weights since the restart);
//   * KKT-based adaptive restarts every check_frequency iterations:
//     candidate = the iterate (current or average) with the smaller
//     omega-weighted KKT error; restart when it fell below 0.2x the value at
//     the last restart (sufficient), below 0.8x and stopped improving
//     (necessary), or when the epoch exceeds 0.36x of all iterations
//     (artificial); at a restart omega <- exp(0.5 log(dy/dx) + 0.5 log omega)
//     from the movement since the previous restart in the scaled norms;
//   * termination on the relative KKT error of the original problem in FP64:
//     ||dist(Ax, [l_r, u_r])||/(1+||b||), ||dual infeasibility||/(1+||c||),
//     |p - d|/(1 + |p| + |d|) all <= tolerance.
//
// FP64 iterative refinement (options.refine = 1, the default).  FP32
// iterates resolve the relative KKT error only to about 1e-6 (rounding the
// exact optimum of a small random LP to FP32 can already leave a 2e-6 gap).
// The solver therefore keeps FP64 master iterates (x_m, y_m) on the device
// and runs the FP32 iteration on the correction (d, e), x = x_m + d,
// y = y_m + e.  The correction problem is the original one translated by
// the master: its FP32 data are the FP64 residuals of the master rounded
// once, A x_m - l_r and A x_m - u_r for the dual update, c + A^T y_m and
// l_x - x_m, u_x - x_m for the primal update (computed by FP64 products with
// the FP32 hi + lo split of the matrix).  At every restart the restart point
// is folded into the master (x_m += d, y_m += e in FP64) and the residuals
// are recomputed, so the FP32 numbers always hold the remaining correction,
// which shrinks with the error: the FP32 resolution applies to the
// correction, not to the answer.  In exact arithmetic the translation
// changes nothing (PDHG commutes with it), so the iteration, the restarts
// and omega are those of the untranslated method; the products inside the
// iteration stay FP32 (8 bytes per non-zero).  This is iterative refinement
// in the sense of Gleixner, Steffy and Wolter (INFORMS J. Computing 2016) —
// FP64 residuals, a correction problem solved in lower precision, an FP64
// update — with one restart epoch of the correction problem per round and
// no rescaling (PDHG's restarts already contract the correction).
#include "adaptive.cuh"
#include "adaptive_kernels.cuh"
#include "pdhg_engine.cuh"

#include <chrono>
#include <cmath>
#include <limits>
#include <vector>

namespace pb {

namespace {

// Deterministic dot product / squared distance: per-block partials (slot
// `slot` of the partial rows), then one block sums them in a fixed order.
//   b != null:             sum a_i b_i
//   b == null:             sum ((a_i - sub_i) / scale_i)^2   (sub, scale may be null)
__global__ void dot_partials_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                    const float* __restrict__ sub, const float* __restrict__ scale,
                                    int n, double* __restrict__ part, int slot) {
    double acc = 0.0;
    PB_GRID_STRIDE(i, n) {
        if (!b) {
            double u = static_cast<double>(a[i]) - (sub ? static_cast<double>(sub[i]) : 0.0);
            if (scale) u /= static_cast<double>(scale[i]);
            acc += u * u;
        } else {
            acc += static_cast<double>(a[i]) * static_cast<double>(b[i]);
        }
    }
    const double v[1] = {acc};
    block_sums_to<1>(v, part, 0, slot);
}




__global__ void reduce_partials_kernel(const double* __restrict__ part, int rows, int slots,
                                       double* __restrict__ out) {
    __shared__ double s_acc[256];
    for (int s = 0; s < slots; ++s) {
        double acc = 0.0;
        for (int r = threadIdx.x; r < rows; r += blockDim.x) acc += part[size_t(r) * kPartSlots + s];
        s_acc[threadIdx.x] = acc;
        __syncthreads();
        for (int w = blockDim.x / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) s_acc[threadIdx.x] += s_acc[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[s] = s_acc[0];
        __syncthreads();
    }
}



__global__ void set_scalars_kernel(float* __restrict__ scal, float primal, float dual) {
    if (blockIdx.x == 0 && threadIdx.x == 0) { scal[0] = primal; scal[1] = dual; }
}









}  // namespace

double PdhgEngine::Kkt::weighted(double omega) const {
    const double gap = pobj - dobj;
    return std::sqrt(omega * omega * pr2 + dr2 / (omega * omega) + gap * gap);
}

void PdhgEngine::setup_adaptive(const pramaan_lp& lp) {
    adaptive_ = true;
    const double sign = lp.obj_sense == PRAMAAN_MAXIMIZE ? -1.0 : 1.0;
    std::vector<double> cmin(static_cast<size_t>(n_));
    double c2 = 0.0;
    for (int j = 0; j < n_; ++j) { cmin[j] = sign * lp.obj_coeffs[j]; c2 += cmin[j] * cmin[j]; }
    c_norm2_ = std::sqrt(c2);
    double b2 = 0.0;
    for (int i = 0; i < m_; ++i) {
        const double lo = lp.row_lower[i], hi = lp.row_upper[i];
        if (lo > -1e29) b2 += lo * lo;
        if (hi < 1e29 && !(lo > -1e29 && lo == hi)) b2 += hi * hi;
    }
    b_norm_ = std::sqrt(b2);
    cmin64_.alloc(n_);
    if (n_) PB_CUDA_CHECK(cudaMemcpyAsync(cmin64_.get(), cmin.data(), size_t(n_) * 8, cudaMemcpyHostToDevice, st_));
    xsum_.alloc(n_); ysum_.alloc(m_);
    xa_.alloc(n_); ya_.alloc(m_);
    if (!opt_.refine) { xl_.alloc(n_); yl_.alloc(m_); }
    xm64_.alloc(n_); ym64_.alloc(m_); actm64_.alloc(m_); rcm64_.alloc(n_); ym32_.alloc(m_);
    rscale_.alloc(m_); cscale_.alloc(n_);
    scal_.alloc(2);
    part_.alloc(size_t(kPartRows) * kPartSlots);
    red_.alloc(kPartSlots);
    PB_CUDA_CHECK(pinned_alloc(&h_red_, sizeof(double) * kPartSlots));
    if (n_) PB_CUDA_CHECK(cudaMemsetAsync(xsum_.get(), 0, xsum_.bytes(), st_));
    if (m_) PB_CUDA_CHECK(cudaMemsetAsync(ysum_.get(), 0, ysum_.bytes(), st_));
    preconditioned_steps();   // replaces the reference steps in tau_ / sigma_
}

// Ruiz + Pock-Chambolle steps (flat operands: called before pack()).
void PdhgEngine::preconditioned_steps() {
    DevBuf<float> r2{static_cast<size_t>(m_ > 0 ? m_ : 1)}, c2{static_cast<size_t>(n_ > 0 ? n_ : 1)};
    if (m_) fill_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rscale_.get(), m_, 1.0f);
    if (n_) fill_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cscale_.get(), n_, 1.0f);
    PB_CUDA_CHECK(cudaGetLastError());
    if (A_.nnz > 0) {
        for (int pass = 0; pass < 10; ++pass) {
            // rows then columns, each against the other side's current scale
            ruiz_pass_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(A_.row_ptr.get(), A_.col.get(), A_.val.get(),
                                                                m_, cscale_.get(), rscale_.get(), r2.get());
            ruiz_pass_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(AT_.row_ptr.get(), AT_.col.get(), AT_.val.get(),
                                                                n_, rscale_.get(), cscale_.get(), c2.get());
            PB_CUDA_CHECK(cudaGetLastError());
            PB_CUDA_CHECK(cudaMemcpyAsync(rscale_.get(), r2.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
            PB_CUDA_CHECK(cudaMemcpyAsync(cscale_.get(), c2.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
        }
    }
    if (m_) pc_step_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(A_.row_ptr.get(), A_.col.get(), A_.val.get(), m_,
                                                             cscale_.get(), rscale_.get(), sigma_.get());
    if (n_) pc_step_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(AT_.row_ptr.get(), AT_.col.get(), AT_.val.get(), n_,
                                                             rscale_.get(), cscale_.get(), tau_.get());
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

// ||Sigma^1/2 A T^1/2||_2 by power iteration on M = T^1/2 A^T Sigma A T^1/2
// (packed operands; Sigma, T the preconditioned steps before eta and omega).
double PdhgEngine::estimate_operator_norm() {
    if (m_ == 0 || n_ == 0 || A_.nnz == 0) return 1.0;
    DevBuf<float> v{static_cast<size_t>(n_)}, t1{static_cast<size_t>(n_)}, u{static_cast<size_t>(m_)},
        w{static_cast<size_t>(n_)}, sqrt_tau{static_cast<size_t>(n_)};
    fill_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(v.get(), n_, float(1.0 / std::sqrt(double(n_))));
    sqrt_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(tau_.get(), n_, sqrt_tau.get());
    PB_CUDA_CHECK(cudaGetLastError());
    double lam = 0.0;
    for (int it = 0; it < 40; ++it) {
        mul_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(v.get(), sqrt_tau.get(), n_, t1.get());
        PB_CUDA_CHECK(cudaGetLastError());
        EpiStoreScaled e1{u.get(), sigma_.get()};          // u = Sigma A T^1/2 v
        SpmvLauncher<EpiStoreScaled, float, float, false>::launch(A_.view(false), t1.get(), e1,
                                                                 status_.get(), st_, dev_);
        EpiStoreScaled e2{w.get(), sqrt_tau.get()};        // w = T^1/2 A^T u = M v
        SpmvLauncher<EpiStoreScaled, float, float, false>::launch(AT_.view(false), u.get(), e2,
                                                                 status_.get(), st_, dev_);
        PB_CUDA_CHECK(cudaMemsetAsync(part_.get(), 0, part_.bytes(), st_));
        dot_partials_kernel<<<256, kThreads, 0, st_>>>(v.get(), w.get(), nullptr, nullptr, n_, part_.get(), 0);
        dot_partials_kernel<<<256, kThreads, 0, st_>>>(w.get(), w.get(), nullptr, nullptr, n_, part_.get(), 1);
        reduce_partials_kernel<<<1, 256, 0, st_>>>(part_.get(), kPartRows, 2, red_.get());
        PB_CUDA_CHECK(cudaGetLastError());
        PB_CUDA_CHECK(cudaMemcpyAsync(h_red_, red_.get(), 16, cudaMemcpyDeviceToHost, st_));
        PB_CUDA_CHECK(cudaStreamSynchronize(st_));
        const double prev = lam;
        lam = h_red_[0];                                   // Rayleigh quotient (||v|| = 1)
        const double wn = std::sqrt(h_red_[1]);
        if (!(wn > 0.0) || !std::isfinite(wn)) break;
        PB_CUDA_CHECK(cudaMemcpyAsync(v.get(), w.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
        scale_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(v.get(), n_, float(1.0 / wn));
        PB_CUDA_CHECK(cudaGetLastError());
        if (it > 5 && std::fabs(lam - prev) <= 1e-4 * std::fabs(lam)) break;
    }
    return lam > 0.0 ? std::sqrt(lam) : 1.0;
}

void PdhgEngine::set_weight(double omega) {
    omega_ = omega;
    set_scalars_kernel<<<1, 1, 0, st_>>>(scal_.get(), float(eta_ / omega), float(eta_ * omega));
    PB_CUDA_CHECK(cudaGetLastError());
}

double PdhgEngine::dist2(const float* a, const float* b, const float* scale, int len) {
    if (len <= 0) return 0.0;
    PB_CUDA_CHECK(cudaMemsetAsync(part_.get(), 0, part_.bytes(), st_));
    dot_partials_kernel<<<256, kThreads, 0, st_>>>(a, nullptr, b, scale, len, part_.get(), 0);
    reduce_partials_kernel<<<1, 256, 0, st_>>>(part_.get(), kPartRows, 1, red_.get());
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaMemcpyAsync(h_red_, red_.get(), 8, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    return h_red_[0];
}

void PdhgEngine::materialize_average() {
    const double inv = avg_count_ > 0 ? 1.0 / double(avg_count_) : 0.0;
    if (avg_count_ > 0) {
        if (n_) average_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(xsum_.get(), n_, inv, xa_.get());
        if (m_) average_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(ysum_.get(), m_, inv, ya_.get());
    } else {
        if (n_) PB_CUDA_CHECK(cudaMemcpyAsync(xa_.get(), x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
        if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(ya_.get(), y_.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
    }
    PB_CUDA_CHECK(cudaGetLastError());
}

// Restart from the average (already materialized in xa_/ya_) or the current
// iterate: x̄ <- x, running sums cleared.
void PdhgEngine::restart_to(bool average) {
    if (average) {
        if (n_) copy2_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(xa_.get(), n_, x_.get(), xbar_.get());
        if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(y_.get(), ya_.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
    } else {
        if (n_) PB_CUDA_CHECK(cudaMemcpyAsync(xbar_.get(), x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
    }
    PB_CUDA_CHECK(cudaGetLastError());
    if (n_) PB_CUDA_CHECK(cudaMemsetAsync(xsum_.get(), 0, xsum_.bytes(), st_));
    if (m_) PB_CUDA_CHECK(cudaMemsetAsync(ysum_.get(), 0, ysum_.bytes(), st_));
    avg_count_ = 0;
}

void PdhgEngine::fold(bool first) {
    if (first) {
        if (n_) init_master_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(vlo64_.get(), vhi64_.get(), n_, xm64_.get());
        if (m_) PB_CUDA_CHECK(cudaMemsetAsync(ym64_.get(), 0, ym64_.bytes(), st_));
        if (n_) PB_CUDA_CHECK(cudaMemsetAsync(x_.get(), 0, size_t(n_) * 4, st_));
        if (n_) PB_CUDA_CHECK(cudaMemsetAsync(xbar_.get(), 0, size_t(n_) * 4, st_));
        if (m_) PB_CUDA_CHECK(cudaMemsetAsync(y_.get(), 0, size_t(m_) * 4, st_));
    } else {
        if (n_) fold_into_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(xm64_.get(), x_.get(), xbar_.get(), n_);
        if (m_) fold_into_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(ym64_.get(), y_.get(), nullptr, m_);
        ++folds_;
    }
    PB_CUDA_CHECK(cudaGetLastError());
    // FP64 residuals of the master (hi + lo matrix values, FP64 accumulation)
    if (m_) {
        EpiStore<double, double> e{actm64_.get()};
        if (A_.has_lo)
            SpmvLauncher<EpiStore<double, double>, double, double, true>::launch(A_.view(true), xm64_.get(), e, status_.get(), st_, dev_);
        else
            SpmvLauncher<EpiStore<double, double>, double, double, false>::launch(A_.view(false), xm64_.get(), e, status_.get(), st_, dev_);
        fold_rows_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rlo64_.get(), rhi64_.get(), actm64_.get(), ym64_.get(), m_,
                                                            lr_.get(), ur_.get(), ym32_.get());
    }
    if (n_) {
        EpiStore<double, double> e{rcm64_.get()};
        if (AT_.has_lo)
            SpmvLauncher<EpiStore<double, double>, double, double, true>::launch(AT_.view(true), ym64_.get(), e, status_.get(), st_, dev_);
        else
            SpmvLauncher<EpiStore<double, double>, double, double, false>::launch(AT_.view(false), ym64_.get(), e, status_.get(), st_, dev_);
        fold_cols_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cmin64_.get(), vlo64_.get(), vhi64_.get(), xm64_.get(), n_,
                                                            rcm64_.get(), c_.get(), lx_.get(), ux_.get());
    }
    PB_CUDA_CHECK(cudaGetLastError());
}

namespace {
void fill_kkt(const double* r, double b_norm, double c_norm, PdhgEngine::Kkt& q) {
    q.pr2 = r[0] + r[4];
    q.dr2 = r[1] + r[5];
    q.dobj = r[2] + r[6];
    q.pobj = r[7];
    q.nonfinite = r[3] > 0.0 || !std::isfinite(q.pr2) || !std::isfinite(q.dr2) ||
                  !std::isfinite(q.pobj) || !std::isfinite(q.dobj);
    q.rel_p = std::sqrt(q.pr2) / (1.0 + b_norm);
    q.rel_d = std::sqrt(q.dr2) / (1.0 + c_norm);
    q.rel_gap = std::fabs(q.pobj - q.dobj) / (1.0 + std::fabs(q.pobj) + std::fabs(q.dobj));
}
}  // namespace

void PdhgEngine::kkt_pair(Kkt& cur, Kkt& avg) {
    materialize_average();
    PB_CUDA_CHECK(cudaMemsetAsync(part_.get(), 0, part_.bytes(), st_));
    const float* xs[2] = {x_.get(), xa_.get()};
    const float* ys[2] = {y_.get(), ya_.get()};
    for (int k = 0; k < 2; ++k) {
        if (m_ > 0) {
            EpiRowKkt er{rlo64_.get(), rhi64_.get(), actm64_.get(), ym64_.get(), ys[k], part_.get(), 8 * k};
            if (A_.has_lo)
                SpmvLauncher<EpiRowKkt, double, float, true>::launch(A_.view(true), xs[k], er, status_.get(), st_, dev_);
            else
                SpmvLauncher<EpiRowKkt, double, float, false>::launch(A_.view(false), xs[k], er, status_.get(), st_, dev_);
        }
        if (n_ > 0) {
            EpiColKkt ec{cmin64_.get(), vlo64_.get(), vhi64_.get(), rcm64_.get(), xm64_.get(), xs[k], part_.get(),
                         8 * k + 4};
            if (AT_.has_lo)
                SpmvLauncher<EpiColKkt, double, float, true>::launch(AT_.view(true), ys[k], ec, status_.get(), st_, dev_);
            else
                SpmvLauncher<EpiColKkt, double, float, false>::launch(AT_.view(false), ys[k], ec, status_.get(), st_, dev_);
        }
    }
    reduce_partials_kernel<<<1, 256, 0, st_>>>(part_.get(), kPartRows, 16, red_.get());
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaMemcpyAsync(h_red_, red_.get(), 16 * 8, cudaMemcpyDeviceToHost, st_));
    check_device_status();   // synchronises
    fill_kkt(h_red_, b_norm_, c_norm2_, cur);
    fill_kkt(h_red_ + 8, b_norm_, c_norm2_, avg);
}

void PdhgEngine::finish_adaptive() {
    x64_.alloc(n_);
    y64_.alloc(m_);
    if (n_) sum_out_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(xm64_.get(), x_.get(), n_, x64_.get());
    if (m_) sum_out_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(ym64_.get(), y_.get(), m_, y64_.get());
    // the FP32 vectors and iterates of the original problem again
    if (n_) {
        restore_cols_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(cmin64_.get(), vlo64_.get(), vhi64_.get(), n_,
                                                               c_.get(), lx_.get(), ux_.get());
        average_kernel<<<grid_1d(n_), kThreads, 0, st_>>>(x64_.get(), n_, 1.0, x_.get());
        PB_CUDA_CHECK(cudaMemcpyAsync(xbar_.get(), x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
    }
    if (m_) {
        restore_rows_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(rlo64_.get(), rhi64_.get(), m_, lr_.get(), ur_.get());
        average_kernel<<<grid_1d(m_), kThreads, 0, st_>>>(y64_.get(), m_, 1.0, y_.get());
    }
    PB_CUDA_CHECK(cudaGetLastError());
    master_out_ = true;
}

void PdhgEngine::solve_adaptive(pramaan_solve_result* res) {
    constexpr double kSufficient = 0.2, kNecessary = 0.8, kArtificial = 0.36;
    const int cf = opt_.check_frequency;
    const int max_it = opt_.max_iterations;
    const double tol = opt_.tolerance;
    const bool refine = opt_.refine != 0;
    int status = PRAMAAN_STATUS_ITERATION_LIMIT;
    folds_ = 0;
    avg_count_ = 0;
    fold(true);
    if (!refine) {
        if (n_) PB_CUDA_CHECK(cudaMemsetAsync(xl_.get(), 0, xl_.bytes(), st_));
        if (m_) PB_CUDA_CHECK(cudaMemsetAsync(yl_.get(), 0, yl_.bytes(), st_));
    }
    Kkt cur, avg;
    kkt_pair(cur, avg);
    double kkt_restart = cur.weighted(omega_);
    double kkt_prev = std::numeric_limits<double>::infinity();
    int last_restart = 0;
    Kkt last = cur;
    int iter = 0;
    if (cur.converged(tol)) status = PRAMAAN_STATUS_OPTIMAL;
    while (status == PRAMAAN_STATUS_ITERATION_LIMIT && iter < max_it) {
        const int chunk = std::min(cf, max_it - iter);
        iterate(chunk);
        iter += chunk;
        avg_count_ += chunk;
        kkt_pair(cur, avg);
        ++res->checks;
        if (cur.nonfinite || avg.nonfinite) { status = PRAMAAN_STATUS_NUMERICAL_FAILURE; break; }
        last = cur;
        if (cur.converged(tol)) { status = PRAMAAN_STATUS_OPTIMAL; break; }
        if (avg.converged(tol)) {
            restart_to(true);
            last = avg;
            status = PRAMAAN_STATUS_OPTIMAL;
            break;
        }
        // ---- adaptive restart ----
        const double kc = cur.weighted(omega_), ka = avg.weighted(omega_);
        const bool use_avg = ka < kc;
        const double kcand = use_avg ? ka : kc;
        const bool restart = kcand <= kSufficient * kkt_restart ||
                             (kcand <= kNecessary * kkt_restart && kcand > kkt_prev) ||
                             (iter - last_restart) >= kArtificial * iter;
        kkt_prev = kcand;
        if (!restart) continue;
        restart_to(use_avg);
        // movement since the previous restart point, in the scaled norms: with
        // refinement the master is that point, so the correction itself
        const double dx = std::sqrt(dist2(x_.get(), refine ? nullptr : xl_.get(), cscale_.get(), n_));
        const double dy = std::sqrt(dist2(y_.get(), refine ? nullptr : yl_.get(), rscale_.get(), m_));
        if (dx > 1e-10 && dy > 1e-10) {
            const double w = std::exp(0.5 * std::log(dy / dx) + 0.5 * std::log(omega_));
            if (std::isfinite(w) && w > 0.0) set_weight(w);
        }
        if (refine) {
            fold(false);
        } else {
            if (n_) PB_CUDA_CHECK(cudaMemcpyAsync(xl_.get(), x_.get(), size_t(n_) * 4, cudaMemcpyDeviceToDevice, st_));
            if (m_) PB_CUDA_CHECK(cudaMemcpyAsync(yl_.get(), y_.get(), size_t(m_) * 4, cudaMemcpyDeviceToDevice, st_));
        }
        kkt_restart = kcand;
        kkt_prev = std::numeric_limits<double>::infinity();
        last_restart = iter;
        ++res->restarts;
    }
    finish_adaptive();
    res->status = status;
    res->iterations = status == PRAMAAN_STATUS_ITERATION_LIMIT ? max_it : iter;
    res->rel_primal = last.rel_p;
    res->rel_dual = last.rel_d;
    res->rel_gap = last.rel_gap;
    res->primal_weight = omega_;
    res->step_size = eta_;
}

}  // namespace pb
