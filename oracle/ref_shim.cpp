// ref_shim.cpp — C entry points over the reference's own solvers, built by
// oracle/build.py against the reference's sources into oracle/_ref/.  Test
// infrastructure only: it lets the parity tests run the unmodified reference
// (RevisedSimplex, DualSimplex, InteriorPointSolver, parse_mps and — with
// REF_WITH_GPU — gpu::PdhgSolver and its test-harness launchers compiled for
// sm_100a) on the same inputs as libpramaan_b200.
#include <cstdint>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#include "pramaan/dual_simplex.hpp"
#include "pramaan/ipm/interior_point.hpp"
#include "pramaan/ir.hpp"
#include "pramaan/mps_parser.hpp"
#include "pramaan/simplex.hpp"
#ifdef REF_WITH_GPU
#include "pramaan/gpu/pdhg_solver.hpp"
namespace pramaan {
namespace gpu {
void launch_spmv(const std::vector<int>&, const std::vector<int>&, const std::vector<float>&,
                 const std::vector<float>&, std::vector<float>&, int, int);
void launch_spmv_t(const std::vector<int>&, const std::vector<int>&, const std::vector<float>&,
                   const std::vector<float>&, std::vector<float>&, int, int);
void launch_pdhg_iteration(float*, float*, const float*, const float*, const float*, int, int,
                           float, float);
}  // namespace gpu
}  // namespace pramaan
#endif

#define REF_API extern "C" __attribute__((visibility("default")))

using namespace pramaan;

struct ref_lp {   // same layout as orc_lp / pramaan_lp
    int32_t m, n, nnz, obj_sense;
    double obj_offset;
    const double* c;
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* values;
    const double* row_lower;
    const double* row_upper;
    const double* var_lower;
    const double* var_upper;
};

struct ref_result {
    int32_t status;
    int32_t iterations;
    int32_t crash_basis_pivots;
    int32_t reserved;
    double primal_residual;
    double dual_residual;
    double objective_value;
    double* x;             // [n] out, written when the solver returned x
    double* row_activity;  // [m] out
};

static thread_local std::string g_err;

static ModelIR to_model(const ref_lp* lp) {
    std::vector<CSRMatrix::Index> rp(lp->row_ptr, lp->row_ptr + lp->m + 1);
    std::vector<CSRMatrix::Index> ci(lp->col_idx, lp->col_idx + lp->nnz);
    std::vector<double> v(lp->values, lp->values + lp->nnz);
    std::vector<std::string> rn(static_cast<size_t>(lp->m)), vn(static_cast<size_t>(lp->n));
    for (int i = 0; i < lp->m; ++i) rn[i] = "r" + std::to_string(i);
    for (int j = 0; j < lp->n; ++j) vn[j] = "x" + std::to_string(j);
    return ModelIR(lp->obj_sense == 1 ? ObjSense::kMaximize : ObjSense::kMinimize, lp->obj_offset,
                   std::vector<double>(lp->c, lp->c + lp->n),
                   CSRMatrix(std::move(rp), std::move(ci), std::move(v), lp->n),
                   std::vector<double>(lp->row_lower, lp->row_lower + lp->m),
                   std::vector<double>(lp->row_upper, lp->row_upper + lp->m), std::move(rn),
                   std::vector<double>(lp->var_lower, lp->var_lower + lp->n),
                   std::vector<double>(lp->var_upper, lp->var_upper + lp->n),
                   std::vector<VarType>(static_cast<size_t>(lp->n), VarType::kContinuous),
                   std::move(vn));
}

static void fill(const SolveResult& r, ref_result* out) {
    out->status = static_cast<int32_t>(r.status);
    out->iterations = r.iterations;
    out->crash_basis_pivots = r.crash_basis_pivots;
    out->primal_residual = r.primal_residual;
    out->dual_residual = r.dual_residual;
    out->objective_value = r.objective_value;
    if (out->x && !r.x.empty()) std::memcpy(out->x, r.x.data(), r.x.size() * sizeof(double));
    if (out->row_activity && !r.row_activity.empty())
        std::memcpy(out->row_activity, r.row_activity.data(), r.row_activity.size() * sizeof(double));
}

template <class F>
static int guarded(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

REF_API const char* ref_last_error() { return g_err.c_str(); }

REF_API int ref_simplex_solve(const ref_lp* lp, int32_t max_iterations, double tolerance,
                              const double* hint, ref_result* out) {
    return guarded([&] {
        RevisedSimplex::Options o;
        o.max_iterations = max_iterations;
        o.tolerance = tolerance;
        if (hint) o.primal_start_hint.assign(hint, hint + lp->n);
        fill(RevisedSimplex(o).solve(to_model(lp)), out);
    });
}

REF_API int ref_dual_simplex_solve(const ref_lp* lp, int32_t max_iterations, double tolerance,
                                   ref_result* out) {
    return guarded([&] {
        DualSimplex::Options o;
        o.max_iterations = max_iterations;
        o.tolerance = tolerance;
        SolveResult r;
        DualSimplex(o).captureBasis(to_model(lp), &r);
        fill(r, out);
    });
}

REF_API int ref_ipm_solve(const ref_lp* lp, int32_t max_iterations, double tolerance,
                          ref_result* out) {
    return guarded([&] {
        InteriorPointSolver::Options o;
        o.max_iterations = max_iterations;
        o.tolerance = tolerance;
        fill(InteriorPointSolver(o).solve(to_model(lp)), out);
    });
}

// MPS loading through the reference parser: ref_mps_open parses and keeps
// the model; ref_mps_dims / ref_mps_fetch copy it out; ref_mps_close frees it.
struct ref_mps {
    ModelIR model;
};

REF_API int ref_mps_open(const char* path, ref_mps** out) {
    return guarded([&] {
        auto h = std::make_unique<ref_mps>();
        h->model = parse_mps(path);
        *out = h.release();
    });
}

REF_API void ref_mps_dims(const ref_mps* h, int32_t* m, int32_t* n, int32_t* nnz, int32_t* sense,
                          double* offset) {
    *m = h->model.numRows();
    *n = h->model.numVars();
    *nnz = h->model.A.nnz();
    *sense = h->model.obj_sense == ObjSense::kMaximize ? 1 : 0;
    *offset = h->model.obj_offset;
}

REF_API void ref_mps_fetch(const ref_mps* h, double* c, int32_t* row_ptr, int32_t* col_idx,
                           double* values, double* row_lower, double* row_upper, double* var_lower,
                           double* var_upper) {
    const ModelIR& M = h->model;
    std::memcpy(c, M.obj_coeffs.data(), M.obj_coeffs.size() * 8);
    std::memcpy(row_ptr, M.A.rowPtr().data(), M.A.rowPtr().size() * 4);
    std::memcpy(col_idx, M.A.colIdx().data(), M.A.colIdx().size() * 4);
    std::memcpy(values, M.A.values().data(), M.A.values().size() * 8);
    std::memcpy(row_lower, M.row_lower.data(), M.row_lower.size() * 8);
    std::memcpy(row_upper, M.row_upper.data(), M.row_upper.size() * 8);
    std::memcpy(var_lower, M.var_lower.data(), M.var_lower.size() * 8);
    std::memcpy(var_upper, M.var_upper.data(), M.var_upper.size() * 8);
}

REF_API void ref_mps_close(ref_mps* h) { delete h; }

#ifdef REF_WITH_GPU
REF_API int ref_pdhg_solve(const ref_lp* lp, double tolerance, int32_t max_iterations,
                           int32_t check_frequency, ref_result* out) {
    return guarded([&] {
        gpu::PdhgOptions o;
        o.tolerance = tolerance;
        o.max_iterations = max_iterations;
        o.check_frequency = check_frequency;
        gpu::PdhgSolver s(o);
        fill(s.solve(to_model(lp)), out);
    });
}

REF_API int ref_launch_spmv(const int32_t* rp, const int32_t* ci, const float* v, int32_t nnz,
                            const float* x, float* y, int32_t m, int32_t n) {
    return guarded([&] {
        std::vector<int> r(rp, rp + m + 1), c(ci, ci + nnz);
        std::vector<float> vv(v, v + nnz), xx(x, x + n), yy;
        gpu::launch_spmv(r, c, vv, xx, yy, m, n);
        if (!yy.empty()) std::memcpy(y, yy.data(), yy.size() * 4);
    });
}

REF_API int ref_launch_spmv_t(const int32_t* rp, const int32_t* ci, const float* v, int32_t nnz,
                              const float* x, float* y, int32_t m, int32_t n) {
    return guarded([&] {
        std::vector<int> r(rp, rp + m + 1), c(ci, ci + nnz);
        std::vector<float> vv(v, v + nnz), xx(x, x + m), yy;
        gpu::launch_spmv_t(r, c, vv, xx, yy, m, n);
        if (!yy.empty()) std::memcpy(y, yy.data(), yy.size() * 4);
    });
}

REF_API int ref_launch_pdhg_iteration(float* x, float* y, const float* g, const float* ax,
                                      const float* b, int32_t n, int32_t m, float tau, float sigma) {
    return guarded([&] { gpu::launch_pdhg_iteration(x, y, g, ax, b, n, m, tau, sigma); });
}
#endif
