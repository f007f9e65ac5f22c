// abi.cu — the extern "C" boundary of libpramaan_b200.so.
//
// Every entry point catches C++ exceptions, records their text in a
// thread-local buffer and returns a negative status, so no exception ever
// crosses the C ABI.
#include <chrono>
#include <cstring>
#include <cmath>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "batch.cuh"
#include "certificate.cuh"
#include "gnn.cuh"
#include "pdhg_engine.cuh"

struct pramaan_pdhg_session {
    std::unique_ptr<pb::PdhgEngine> eng;
};
struct pramaan_gnn {
    int device = 0;
    std::unique_ptr<pb::GnnModel> model;
};
struct pramaan_gnn_graph {
    std::unique_ptr<pb::GnnGraph> graph;
};

namespace pb {
// noalloc.cu
void spmv_noalloc(const int32_t* d_row_ptr, const int32_t* d_col_idx, const float* d_values,
                  int32_t m, int32_t n, int32_t nnz, const float* d_x, float* d_y,
                  cudaStream_t stream);
// ceiling.cu
double measure_gather_rate(const float* d_x, int n, bool cached, int reps);
}  // namespace pb

namespace pb {
namespace {

thread_local std::string g_last_error;

template <class F>
int guarded(F&& fn) {
    try {
        fn();
        g_last_error.clear();
        return PRAMAAN_OK;
    } catch (const InvalidArgument& e) {
        g_last_error = e.what();
        return PRAMAAN_ERR_INVALID_ARGUMENT;
    } catch (const DeviceTimeout& e) {
        g_last_error = e.what();
        return PRAMAAN_ERR_DEVICE_TIMEOUT;
    } catch (const CudaError& e) {
        g_last_error = e.what();
        return PRAMAAN_ERR_CUDA;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return PRAMAAN_ERR_INTERNAL;
    } catch (...) {
        g_last_error = "unknown exception";
        return PRAMAAN_ERR_INTERNAL;
    }
}

constexpr int kThreads = 256;

// Step-1 dense iteration (src/gpu/pdhg.cu:42-66): nvcc contracts both
// reference expressions to one FMA each; written explicitly here.
__global__ void step1_kernel(float* __restrict__ x, const float* __restrict__ g, int n, float tau,
                             float* __restrict__ y, const float* __restrict__ ax,
                             const float* __restrict__ b, int m, float sigma) {
    const int total = n > m ? n : m;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        if (i < n) x[i] = fmaxf(0.0f, __fmaf_rn(-tau, g[i], x[i]));
        if (i < m) y[i] = __fmaf_rn(sigma, __fsub_rn(ax[i], b[i]), y[i]);
    }
}

struct StreamHolder {
    cudaStream_t st = nullptr;
    StreamHolder() { PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)); }
    ~StreamHolder() { if (st) cudaStreamDestroy(st); }
};

void check_flag(int* d_flag, cudaStream_t st) {
    int h = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&h, d_flag, 4, cudaMemcpyDeviceToHost, st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
    if (h & 1) throw InvalidArgument("row_ptr must start at 0, be non-decreasing and end at nnz");
    if (h & 2) throw InvalidArgument("col_idx entry out of bounds");
}

void spmv_harness(const int32_t* row_ptr, const int32_t* col_idx, const float* values, int nnz,
                  const float* x, float* y_out, int m, int n, bool transpose) {
    if (m < 0 || n < 0 || nnz < 0) throw InvalidArgument("negative dimension");
    const int out_len = transpose ? n : m;
    const int in_len = transpose ? m : n;
    if (out_len == 0) return;
    if (!y_out) throw InvalidArgument("y_out is NULL");
    if (m > 0 && !row_ptr) throw InvalidArgument("row_ptr is NULL");
    if (nnz > 0 && (!col_idx || !values)) throw InvalidArgument("col_idx/values is NULL");
    if (in_len > 0 && nnz > 0 && !x) throw InvalidArgument("x is NULL");
    StreamHolder sh;
    cudaStream_t st = sh.st;
    int dev = 0;
    PB_CUDA_CHECK(cudaGetDevice(&dev));
    DevBuf<int> flag(1);
    PB_CUDA_CHECK(cudaMemsetAsync(flag.get(), 0, 4, st));
    CsrDevice A;
    static const int zero_rp = 0;
    csr_upload_f32(A, m, n, nnz, m > 0 ? row_ptr : &zero_rp, col_idx, values, st, flag.get());
    check_flag(flag.get(), st);
    DevBuf<float> dx{size_t(in_len > 0 ? in_len : 1)}, dy{size_t(out_len)};
    if (in_len > 0 && x)
        PB_CUDA_CHECK(cudaMemcpyAsync(dx.get(), x, size_t(in_len) * 4, cudaMemcpyHostToDevice, st));
    else
        PB_CUDA_CHECK(cudaMemsetAsync(dx.get(), 0, dx.bytes(), st));
    EpiStore<float, float> epi{dy.get()};
    SpmvLauncher<EpiStore<float, float>, float, float, false>::blocks_per_sm(dev);
    if (!transpose) {
        A.pack(st);
        SpmvLauncher<EpiStore<float, float>, float, float, false>::launch(A.view(false), dx.get(), epi,
                                                                         flag.get(), st, dev);
    } else {
        CsrDevice AT;
        csr_transpose(A, AT, st);
        AT.pack(st);
        SpmvLauncher<EpiStore<float, float>, float, float, false>::launch(AT.view(false), dx.get(),
                                                                         epi, flag.get(), st, dev);
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    PB_CUDA_CHECK(cudaMemcpyAsync(y_out, dy.get(), size_t(out_len) * 4, cudaMemcpyDeviceToHost, st));
    int h_status = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&h_status, flag.get(), 4, cudaMemcpyDeviceToHost, st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
    if (h_status & kDevErrTimeout) throw DeviceTimeout("device wait on a bulk copy exceeded its time limit");
}

pramaan_pdhg_options defaults() {
    pramaan_pdhg_options o;
    std::memset(&o, 0, sizeof(o));
    o.tolerance = 1e-6;
    o.max_iterations = 100000;
    o.check_frequency = 100;
    o.algorithm = PRAMAAN_ALGO_REFERENCE;
    o.termination = PRAMAAN_TERM_REFERENCE;
    o.device = 0;
    o.use_graph = 1;
    o.profile_kernels = 0;
    o.refine = 1;
    o.reserved_d = 0.0;
    return o;
}

// Re-raises the failure of a nested entry point with its own text.
[[noreturn]] void throw_last(int rc) {
    const std::string msg = g_last_error;
    if (rc == PRAMAAN_ERR_INVALID_ARGUMENT) throw InvalidArgument(msg);
    if (rc == PRAMAAN_ERR_DEVICE_TIMEOUT) throw DeviceTimeout(msg);
    if (rc == PRAMAAN_ERR_CUDA) throw CudaError(msg);
    throw std::runtime_error(msg);
}

void same_device(const pramaan_gnn* net, const pramaan_gnn_graph* gr) {
    if (!net || !gr) throw InvalidArgument("net and graph must not be NULL");
    if (net->device != gr->graph->device) throw InvalidArgument("net and graph live on different devices");
}

}  // namespace
}  // namespace pb

using namespace pb;

extern "C" {

const char* pramaan_version(void) { return "pramaan_b200 0.1.0 (sm_100a)"; }

const char* pramaan_last_error(void) { return g_last_error.c_str(); }

void pramaan_pdhg_default_options(pramaan_pdhg_options* opt) {
    if (opt) *opt = defaults();
}

int pramaan_pdhg_solve_batch(const pramaan_lp* lps, int32_t count, const pramaan_pdhg_options* opt,
                             pramaan_solve_result* results) {
    return pramaan_pdhg_solve_batch_warm(lps, count, opt, nullptr, results);
}

int pramaan_pdhg_solve_batch_warm(const pramaan_lp* lps, int32_t count, const pramaan_pdhg_options* opt,
                                  const pramaan_warm_start* warm, pramaan_solve_result* results) {
    return guarded([&] {
        if (count < 0) throw InvalidArgument("count must be >= 0");
        if (count > 0 && (!lps || !results)) throw InvalidArgument("lps and results must not be NULL");
        pramaan_pdhg_options o = opt ? *opt : defaults();
        if (!opt) {
            o.algorithm = PRAMAAN_ALGO_HALPERN;
            o.termination = PRAMAAN_TERM_RELATIVE_KKT;
        }
        DeviceGuard g(o.device);
        AdaptiveBatch batch(lps, count, o, warm);
        batch.solve(lps, results);
    });
}

int pramaan_pdhg_solve(const pramaan_lp* lp, const pramaan_pdhg_options* opt,
                       pramaan_solve_result* res) {
    return guarded([&] {
        if (!lp || !res) throw InvalidArgument("lp and result must not be NULL");
        const pramaan_pdhg_options o = opt ? *opt : defaults();
        const auto t0 = std::chrono::steady_clock::now();
        res->status = PRAMAAN_STATUS_ITERATION_LIMIT;
        res->iterations = 0;
        res->restarts = 0;
        res->checks = 0;
        res->compactions = 0.0;
        res->primal_residual = std::numeric_limits<double>::infinity();
        res->dual_residual = std::numeric_limits<double>::infinity();
        res->objective_value = 0.0;
        validate_lp(*lp);
        validate_options(o);
        const int m = lp->num_rows, n = lp->num_cols;
        // Trivial: no variables (src/gpu/pdhg_solver.cu:179-184).
        if (n == 0) {
            res->status = PRAMAAN_STATUS_OPTIMAL;
            res->objective_value = lp->obj_offset;
            if (res->row_activity)
                for (int i = 0; i < m; ++i) res->row_activity[i] = 0.0;
            res->solve_ms = 0.0;
            return;
        }
        // Guard: NaN/Inf in the objective (src/gpu/pdhg_solver.cu:187-192).
        for (int j = 0; j < n; ++j) {
            if (!std::isfinite(lp->obj_coeffs[j])) {
                res->status = PRAMAAN_STATUS_NUMERICAL_FAILURE;
                res->solve_ms = 0.0;
                return;
            }
        }
        DeviceGuard g(o.device);
        if (o.algorithm == PRAMAAN_ALGO_HALPERN) {
            // the Halpern iteration lives in the batched engine: a batch of one
            AdaptiveBatch one(lp, 1, o);
            one.solve(lp, res);
            res->compactions = 0.0;
        } else {
            PdhgEngine eng(*lp, o);
            eng.solve(*lp, res);
        }
        res->solve_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

int pramaan_launch_spmv(const int32_t* row_ptr, const int32_t* col_idx, const float* values,
                        int32_t nnz, const float* x, float* y_out, int32_t m, int32_t n) {
    return guarded([&] { spmv_harness(row_ptr, col_idx, values, nnz, x, y_out, m, n, false); });
}

int pramaan_launch_spmv_t(const int32_t* row_ptr, const int32_t* col_idx, const float* values,
                          int32_t nnz, const float* x, float* y_out, int32_t m, int32_t n) {
    return guarded([&] {
        if (m == 0 && n > 0 && y_out)
            for (int j = 0; j < n; ++j) y_out[j] = 0.0f;
        if (m == 0) return;
        spmv_harness(row_ptr, col_idx, values, nnz, x, y_out, m, n, true);
    });
}

int pramaan_launch_pdhg_iteration(float* h_x, float* h_y, const float* h_gradient,
                                  const float* h_Ax_bar, const float* h_b, int32_t n, int32_t m,
                                  float tau, float sigma) {
    return guarded([&] {
        if (n <= 0 && m <= 0) return;
        if (n < 0) n = 0;
        if (m < 0) m = 0;
        if (n > 0 && (!h_x || !h_gradient)) throw InvalidArgument("x/gradient is NULL");
        if (m > 0 && (!h_y || !h_Ax_bar || !h_b)) throw InvalidArgument("y/Ax_bar/b is NULL");
        StreamHolder sh;
        cudaStream_t st = sh.st;
        DevBuf<float> dx{size_t(n)}, dg{size_t(n)}, dy{size_t(m)}, dax{size_t(m)}, db{size_t(m)};
        if (n > 0) {
            PB_CUDA_CHECK(cudaMemcpyAsync(dx.get(), h_x, size_t(n) * 4, cudaMemcpyHostToDevice, st));
            PB_CUDA_CHECK(cudaMemcpyAsync(dg.get(), h_gradient, size_t(n) * 4, cudaMemcpyHostToDevice, st));
        }
        if (m > 0) {
            PB_CUDA_CHECK(cudaMemcpyAsync(dy.get(), h_y, size_t(m) * 4, cudaMemcpyHostToDevice, st));
            PB_CUDA_CHECK(cudaMemcpyAsync(dax.get(), h_Ax_bar, size_t(m) * 4, cudaMemcpyHostToDevice, st));
            PB_CUDA_CHECK(cudaMemcpyAsync(db.get(), h_b, size_t(m) * 4, cudaMemcpyHostToDevice, st));
        }
        const int total = n > m ? n : m;
        const int grid = (total + kThreads - 1) / kThreads;
        step1_kernel<<<grid, kThreads, 0, st>>>(dx.get(), dg.get(), n, tau, dy.get(), dax.get(),
                                                 db.get(), m, sigma);
        PB_CUDA_CHECK(cudaGetLastError());
        if (n > 0) PB_CUDA_CHECK(cudaMemcpyAsync(h_x, dx.get(), size_t(n) * 4, cudaMemcpyDeviceToHost, st));
        if (m > 0) PB_CUDA_CHECK(cudaMemcpyAsync(h_y, dy.get(), size_t(m) * 4, cudaMemcpyDeviceToHost, st));
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
    });
}

int pramaan_spmv_noalloc(const int32_t* d_row_ptr, const int32_t* d_col_idx, const float* d_values,
                         int32_t m, int32_t n, int32_t nnz, const float* d_x, float* d_y,
                         void* stream) {
    return guarded([&] {
        spmv_noalloc(d_row_ptr, d_col_idx, d_values, m, n, nnz, d_x, d_y,
                     static_cast<cudaStream_t>(stream));
    });
}

int pramaan_session_create(const pramaan_lp* lp, const pramaan_pdhg_options* opt,
                           pramaan_pdhg_session** out) {
    return guarded([&] {
        if (!lp || !out) throw InvalidArgument("lp and out must not be NULL");
        *out = nullptr;
        const pramaan_pdhg_options o = opt ? *opt : defaults();
        if (o.algorithm != PRAMAAN_ALGO_REFERENCE)
            throw InvalidArgument("sessions step the reference iteration (PRAMAAN_ALGO_REFERENCE)");
        DeviceGuard g(o.device);
        auto s = std::make_unique<pramaan_pdhg_session>();
        s->eng = std::make_unique<PdhgEngine>(*lp, o);
        *out = s.release();
    });
}

int pramaan_session_destroy(pramaan_pdhg_session* s) {
    return guarded([&] {
        if (!s) return;
        DeviceGuard g(s->eng->device());
        delete s;
    });
}

int pramaan_session_iterate(pramaan_pdhg_session* s, int32_t iterations) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        DeviceGuard g(s->eng->device());
        s->eng->iterate(iterations);
    });
}

int pramaan_session_synchronize(pramaan_pdhg_session* s) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        DeviceGuard g(s->eng->device());
        s->eng->synchronize();
    });
}

int pramaan_session_residuals(pramaan_pdhg_session* s, double* primal, double* dual) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        DeviceGuard g(s->eng->device());
        double pv = 0, dv = 0;
        bool nf = false;
        s->eng->residuals(pv, dv, nf);
        if (primal) *primal = nf ? std::numeric_limits<double>::quiet_NaN() : pv;
        if (dual) *dual = nf ? std::numeric_limits<double>::quiet_NaN() : dv;
    });
}

int pramaan_session_get_iterates(pramaan_pdhg_session* s, float* x, float* y) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        DeviceGuard g(s->eng->device());
        s->eng->get_iterates(x, y);
    });
}

void* pramaan_session_stream(pramaan_pdhg_session* s) {
    return s ? static_cast<void*>(s->eng->stream()) : nullptr;
}

int pramaan_session_kernel_times(pramaan_pdhg_session* s, double* ms_dual, double* ms_primal,
                                 int64_t* launches, int32_t reset) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        DeviceGuard g(s->eng->device());
        long long l = 0;
        s->eng->kernel_times(ms_dual, ms_primal, &l, reset != 0);
        if (launches) *launches = l;
    });
}

int pramaan_session_kernel_bytes(pramaan_pdhg_session* s, double* bytes_dual, double* bytes_primal) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        if (bytes_dual) *bytes_dual = s->eng->bytes_dual();
        if (bytes_primal) *bytes_primal = s->eng->bytes_primal();
    });
}

int pramaan_session_gather_info(pramaan_pdhg_session* s, int32_t* slots_dual, int32_t* slots_primal,
                                int32_t* l1_dual, int32_t* l1_primal, int32_t* blocks_dual,
                                int32_t* blocks_primal) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        if (slots_dual) *slots_dual = s->eng->hot_slots_dual();
        if (slots_primal) *slots_primal = s->eng->hot_slots_primal();
        if (l1_dual) *l1_dual = s->eng->gather_l1_dual();
        if (l1_primal) *l1_primal = s->eng->gather_l1_primal();
        if (blocks_dual) *blocks_dual = s->eng->blocks_dual();
        if (blocks_primal) *blocks_primal = s->eng->blocks_primal();
    });
}

int pramaan_session_panel_info(pramaan_pdhg_session* s, int32_t* panels, int32_t* long_rows, int64_t* long_nnz,
                               int32_t* min_len, int32_t* hot_rows, int64_t* hot_nnz) {
    return guarded([&] {
        if (!s) throw InvalidArgument("session is NULL");
        int p = 0, l = 0, ml = 0, hr = 0;
        long long nz = 0, hz = 0;
        s->eng->panel_info(&p, &l, &nz, &ml, &hr, &hz);
        if (panels) *panels = p;
        if (long_rows) *long_rows = l;
        if (long_nnz) *long_nnz = nz;
        if (min_len) *min_len = ml;
        if (hot_rows) *hot_rows = hr;
        if (hot_nnz) *hot_nnz = hz;
    });
}

int pramaan_measure_gather_rate(const float* d_x, int32_t n, int32_t cached, int32_t reps,
                                double* gathers_per_s) {
    return guarded([&] {
        if (!gathers_per_s) throw InvalidArgument("gathers_per_s must not be NULL");
        *gathers_per_s = measure_gather_rate(d_x, n, cached != 0, reps);
    });
}

int pramaan_release_cached_memory(int32_t device) {
    return guarded([&] {
        if (device < -1) throw InvalidArgument("device must be -1 or a device ordinal");
        device_cache_release(device);
    });
}

// ---- precision ladder ----------------------------------------------------

void pramaan_ladder_default_options(pramaan_ladder_options* opt) {
    if (!opt) return;
    std::memset(opt, 0, sizeof(*opt));
    opt->residual_threshold = 1e-6;
    opt->gpu_max_iterations = 100000;
    opt->gpu_check_frequency = 100;
    opt->gpu_tolerance = 1e-6;
    opt->refine = 1;
    opt->refine_max_iterations = 400000;
    opt->refine_tolerance = 1e-9;
    opt->device = 0;
}

namespace {
// The reference gate (src/gpu/precision_ladder.cpp:91-121): accept iff
// optimal and both residuals <= T; otherwise the escalation reason.
int ladder_gate(const pramaan_solve_result& r, double T) {
    if (r.status == PRAMAAN_STATUS_OPTIMAL) {
        if (r.primal_residual <= T && r.dual_residual <= T) return PRAMAAN_ESCALATION_NONE;
        return r.primal_residual > T ? PRAMAAN_ESCALATION_HIGH_PRIMAL_RESIDUAL : PRAMAAN_ESCALATION_HIGH_DUAL_RESIDUAL;
    }
    if (r.status == PRAMAAN_STATUS_ITERATION_LIMIT) return PRAMAAN_ESCALATION_GPU_ITERATION_LIMIT;
    if (r.status == PRAMAAN_STATUS_NUMERICAL_FAILURE) return PRAMAAN_ESCALATION_GPU_NUMERICAL_FAILURE;
    return PRAMAAN_ESCALATION_GPU_NOT_OPTIMAL;
}
}  // namespace

int pramaan_ladder_solve(const pramaan_lp* lp, const pramaan_ladder_options* opt, pramaan_ladder_result* out) {
    return guarded([&] {
        if (!lp || !out) throw InvalidArgument("lp and result must not be NULL");
        pramaan_ladder_options o;
        pramaan_ladder_default_options(&o);
        if (opt) o = *opt;
        const auto t0 = std::chrono::steady_clock::now();
        const int n = lp->num_cols, m = lp->num_rows;
        std::vector<double> x1(size_t(n > 0 ? n : 1)), y1(size_t(m > 0 ? m : 1)), a1(size_t(m > 0 ? m : 1));
        // ---- rung 1: the reference FP32 PDHG ----
        pramaan_pdhg_options g = defaults();
        g.tolerance = o.gpu_tolerance;
        g.max_iterations = o.gpu_max_iterations;
        g.check_frequency = o.gpu_check_frequency;
        g.device = o.device;
        pramaan_solve_result r1{};
        r1.x = x1.data(); r1.y = y1.data(); r1.row_activity = a1.data();
        const int rc1 = pramaan_pdhg_solve(lp, &g, &r1);
        if (rc1 != PRAMAAN_OK) throw_last(rc1);
        out->gpu_status = r1.status;
        out->gpu_iterations = r1.iterations;
        out->gpu_primal_residual = r1.primal_residual;
        out->gpu_dual_residual = r1.dual_residual;
        out->gpu_objective = r1.objective_value;
        out->gpu_elapsed_ms = r1.solve_ms;
        out->escalation_reason = ladder_gate(r1, o.residual_threshold);
        out->refine_escalation_reason = PRAMAAN_ESCALATION_NONE;
        out->refine_status = PRAMAAN_STATUS_ITERATION_LIMIT;
        out->refine_iterations = 0;
        out->refine_primal_residual = out->refine_dual_residual = std::numeric_limits<double>::infinity();
        out->refine_objective = 0.0;
        out->refine_elapsed_ms = 0.0;
        const pramaan_solve_result* best = &r1;
        pramaan_solve_result r2{};
        std::vector<double> x2, y2, a2;
        if (out->escalation_reason == PRAMAAN_ESCALATION_NONE) {
            out->stage = PRAMAAN_LADDER_GPU_FP32;
        } else if (o.refine) {
            // ---- rung 2: FP64 refinement on the GPU ----
            x2.resize(x1.size()); y2.resize(y1.size()); a2.resize(a1.size());
            pramaan_pdhg_options g2 = defaults();
            g2.algorithm = PRAMAAN_ALGO_ADAPTIVE;
            g2.termination = PRAMAAN_TERM_RELATIVE_KKT;
            g2.refine = 1;
            g2.tolerance = o.refine_tolerance;
            g2.max_iterations = o.refine_max_iterations;
            g2.check_frequency = 64;
            g2.device = o.device;
            r2.x = x2.data(); r2.y = y2.data(); r2.row_activity = a2.data();
            const int rc2 = pramaan_pdhg_solve(lp, &g2, &r2);
            if (rc2 != PRAMAAN_OK) throw_last(rc2);
            out->refine_status = r2.status;
            out->refine_iterations = r2.iterations;
            out->refine_primal_residual = r2.primal_residual;
            out->refine_dual_residual = r2.dual_residual;
            out->refine_objective = r2.objective_value;
            out->refine_elapsed_ms = r2.solve_ms;
            out->refine_escalation_reason = ladder_gate(r2, o.residual_threshold);
            const bool better = r2.status == PRAMAAN_STATUS_OPTIMAL &&
                                std::max(r2.primal_residual, r2.dual_residual) <=
                                    std::max(r1.primal_residual, r1.dual_residual);
            if (out->refine_escalation_reason == PRAMAAN_ESCALATION_NONE || better) best = &r2;
            out->stage = out->refine_escalation_reason == PRAMAAN_ESCALATION_NONE ? PRAMAAN_LADDER_GPU_FP64_REFINED
                                                                                : PRAMAAN_LADDER_ESCALATE;
        } else {
            out->stage = PRAMAAN_LADDER_ESCALATE;
        }
        out->rel_primal = best->rel_primal;
        out->rel_dual = best->rel_dual;
        out->rel_gap = best->rel_gap;
        out->objective_value = best->objective_value;
        if (out->x && n > 0) std::memcpy(out->x, best->x, size_t(n) * 8);
        if (out->y && m > 0) std::memcpy(out->y, best->y, size_t(m) * 8);
        if (out->row_activity && m > 0) std::memcpy(out->row_activity, best->row_activity, size_t(m) * 8);
        out->total_elapsed_ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    });
}

// ---- certificates --------------------------------------------------------

int pramaan_certify_batch(const pramaan_lp* lps, int32_t count, const pramaan_warm_start* points,
                          int32_t num_points, int32_t device, pramaan_certificate* out) {
    return guarded([&] {
        if (count < 0 || num_points < 0) throw InvalidArgument("count and num_points must be >= 0");
        if (count == 0 || num_points == 0) return;
        if (!lps || !points || !out) throw InvalidArgument("lps, points and out must not be NULL");
        DeviceGuard g(device);
        CertificateBatch cb(lps, count, device);
        for (int p = 0; p < num_points; ++p) cb.evaluate(points + size_t(p) * count, out + size_t(p) * count);
    });
}

// ---- learned warm start --------------------------------------------------

int32_t pramaan_gnn_num_params(void) { return pb::GnnModel::num_params(); }

int pramaan_gnn_create(int32_t device, uint64_t seed, pramaan_gnn** out) {
    return guarded([&] {
        if (!out) throw InvalidArgument("out is NULL");
        *out = nullptr;
        DeviceGuard g(device);
        auto n = std::make_unique<pramaan_gnn>();
        n->device = device;
        n->model = std::make_unique<GnnModel>(device, seed);
        *out = n.release();
    });
}

int pramaan_gnn_destroy(pramaan_gnn* net) {
    return guarded([&] {
        if (!net) return;
        DeviceGuard g(net->device);
        delete net;
    });
}

int pramaan_gnn_get_params(const pramaan_gnn* net, float* params) {
    return guarded([&] {
        if (!net || !params) throw InvalidArgument("net and params must not be NULL");
        DeviceGuard g(net->device);
        net->model->get_params(params);
    });
}

int pramaan_gnn_set_params(pramaan_gnn* net, const float* params) {
    return guarded([&] {
        if (!net || !params) throw InvalidArgument("net and params must not be NULL");
        DeviceGuard g(net->device);
        net->model->set_params(params);
    });
}

int pramaan_gnn_graph_create(const pramaan_lp* lps, int32_t count, const pramaan_warm_start* hints,
                             const pramaan_warm_start* targets, int32_t device, pramaan_gnn_graph** out) {
    return guarded([&] {
        if (!out) throw InvalidArgument("out is NULL");
        *out = nullptr;
        if (count < 0) throw InvalidArgument("count must be >= 0");
        if (count > 0 && !lps) throw InvalidArgument("lps is NULL");
        DeviceGuard g(device);
        auto h = std::make_unique<pramaan_gnn_graph>();
        h->graph = std::make_unique<GnnGraph>(lps, count, hints, targets, device);
        *out = h.release();
    });
}

int pramaan_gnn_graph_destroy(pramaan_gnn_graph* gr) {
    return guarded([&] {
        if (!gr) return;
        DeviceGuard g(gr->graph->device);
        delete gr;
    });
}

int pramaan_gnn_predict(pramaan_gnn* net, const pramaan_gnn_graph* gr, double* const* x_out,
                        double* const* y_out, double* omega_out) {
    return guarded([&] {
        same_device(net, gr);
        DeviceGuard g(net->device);
        net->model->forward(*gr->graph);
        net->model->predict(*gr->graph, x_out, y_out, omega_out);
    });
}

int pramaan_gnn_gradients(pramaan_gnn* net, const pramaan_gnn_graph* gr, float* grad, double* loss) {
    return guarded([&] {
        same_device(net, gr);
        DeviceGuard g(net->device);
        net->model->forward(*gr->graph);
        const double l = net->model->backward(*gr->graph, true);
        if (loss) *loss = l;
        if (grad) net->model->copy_grad(grad);
    });
}

int pramaan_gnn_train_step(pramaan_gnn* net, const pramaan_gnn_graph* gr, float learning_rate, double* loss) {
    return guarded([&] {
        same_device(net, gr);
        if (!(learning_rate > 0.0f) || !std::isfinite(learning_rate))
            throw InvalidArgument("learning_rate must be positive and finite");
        DeviceGuard g(net->device);
        net->model->forward(*gr->graph);
        const double l = net->model->backward(*gr->graph, true);
        net->model->adam_step(learning_rate);
        if (loss) *loss = l;
    });
}

int64_t pramaan_gnn_trace_size(const pramaan_gnn_graph* gr) {
    if (!gr) return 0;
    const pb::GnnGraph& g = *gr->graph;
    return int64_t(pb::kGnnLayers) * (int64_t(g.m) + g.n) * 128 + (int64_t(g.m) + g.n) * 64 + g.n + g.m +
           int64_t(g.K) * 129;
}

int pramaan_gnn_forward_trace(pramaan_gnn* net, const pramaan_gnn_graph* gr, float* out) {
    return guarded([&] {
        same_device(net, gr);
        if (!out) throw InvalidArgument("out is NULL");
        DeviceGuard g(net->device);
        net->model->forward(*gr->graph);
        net->model->trace(*gr->graph, out);
    });
}

}  // extern "C"
