// facade/pdhg_solver.cpp — drop-in replacement for PRAMAAN's
// src/gpu/pdhg_solver.cu and src/gpu/pdhg.cu.
//
// Compiled inside a PRAMAAN tree (it includes the reference's public headers
// pramaan/gpu/pdhg_solver.hpp, pramaan/ir.hpp and pramaan/simplex.hpp) and
// linked against libpramaan_b200.so.  It provides, with the reference's C++
// linkage and semantics:
//   * pramaan::gpu::PdhgSolver::{PdhgSolver, ~PdhgSolver, solve}
//     (include/pramaan/gpu/pdhg_solver.hpp:15-24);
//   * the test-harness launchers launch_spmv, launch_spmv_t and
//     launch_pdhg_iteration (src/gpu/pdhg.cu:77-241) that
//     tests/test_gpu_pdhg.cpp:124-142 and tests/test_pdhg_kernel.cpp:11-17
//     forward-declare.
// Errors: a failed CUDA call surfaces as std::runtime_error("CUDA error in
// <file>:<line> - <msg>") exactly as CUDA_CHECK raises it
// (src/gpu/cuda_utils.cuh:8-15); rejected inputs as std::invalid_argument.
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "pramaan/gpu/pdhg_solver.hpp"
#include "pramaan_b200.h"

namespace pramaan {
namespace gpu {

namespace {

[[noreturn]] void raise_status(int rc) {
    const std::string msg = pramaan_last_error();
    if (rc == PRAMAAN_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

}  // namespace

PdhgSolver::PdhgSolver(const PdhgOptions& options) : options_(options) {}
PdhgSolver::~PdhgSolver() {}

SolveResult PdhgSolver::solve(const ModelIR& model) {
    const int m = static_cast<int>(model.numRows());
    const int n = static_cast<int>(model.numVars());
    SolveResult result;
    result.status = SolveStatus::kIterationLimit;
    result.iterations = 0;

    // The two early returns of the reference keep x empty.
    if (n == 0) {
        result.status = SolveStatus::kOptimal;
        result.objective_value = model.obj_offset;
        result.row_activity.assign(static_cast<size_t>(m), 0.0);
        return result;
    }
    for (int j = 0; j < n; ++j) {
        if (!std::isfinite(model.obj_coeffs[j])) {
            result.status = SolveStatus::kNumericalFailure;
            return result;
        }
    }

    pramaan_lp lp{};
    lp.num_rows = m;
    lp.num_cols = n;
    lp.nnz = static_cast<int32_t>(model.A.nnz());
    lp.obj_sense = model.obj_sense == ObjSense::kMaximize ? PRAMAAN_MAXIMIZE : PRAMAAN_MINIMIZE;
    lp.obj_offset = model.obj_offset;
    lp.obj_coeffs = model.obj_coeffs.data();
    lp.row_ptr = model.A.rowPtr().data();
    lp.col_idx = model.A.colIdx().data();
    lp.values = model.A.values().data();
    lp.row_lower = model.row_lower.data();
    lp.row_upper = model.row_upper.data();
    lp.var_lower = model.var_lower.data();
    lp.var_upper = model.var_upper.data();

    pramaan_pdhg_options opt;
    pramaan_pdhg_default_options(&opt);
    opt.tolerance = options_.tolerance;
    opt.max_iterations = options_.max_iterations;
    opt.check_frequency = options_.check_frequency;

    result.x.assign(static_cast<size_t>(n), 0.0);
    result.row_activity.assign(static_cast<size_t>(m), 0.0);
    pramaan_solve_result r{};
    r.x = result.x.data();
    r.row_activity = result.row_activity.data();
    const int rc = pramaan_pdhg_solve(&lp, &opt, &r);
    if (rc != PRAMAAN_OK) raise_status(rc);

    result.status = static_cast<SolveStatus>(r.status);
    result.iterations = r.iterations;
    result.primal_residual = r.primal_residual;
    result.dual_residual = r.dual_residual;
    result.objective_value = r.objective_value;
    return result;
}

void launch_spmv(const std::vector<int>& row_ptr, const std::vector<int>& col_idx,
                 const std::vector<float>& values, const std::vector<float>& x,
                 std::vector<float>& y_out, int m, int n) {
    if (m == 0) { y_out.clear(); return; }
    y_out.resize(static_cast<size_t>(m));
    const int rc = pramaan_launch_spmv(row_ptr.data(), col_idx.data(), values.data(),
                                       static_cast<int32_t>(values.size()), x.data(),
                                       y_out.data(), m, n);
    if (rc != PRAMAAN_OK) raise_status(rc);
}

void launch_spmv_t(const std::vector<int>& row_ptr, const std::vector<int>& col_idx,
                   const std::vector<float>& values, const std::vector<float>& x,
                   std::vector<float>& y_out, int m, int n) {
    y_out.assign(static_cast<size_t>(n), 0.0f);
    if (n == 0) return;
    const int rc = pramaan_launch_spmv_t(row_ptr.data(), col_idx.data(), values.data(),
                                         static_cast<int32_t>(values.size()), x.data(),
                                         y_out.data(), m, n);
    if (rc != PRAMAAN_OK) raise_status(rc);
}

void launch_pdhg_iteration(float* h_x, float* h_y, const float* h_gradient, const float* h_Ax_bar,
                           const float* h_b, const int n, const int m, const float tau,
                           const float sigma) {
    const int rc = pramaan_launch_pdhg_iteration(h_x, h_y, h_gradient, h_Ax_bar, h_b, n, m, tau,
                                                 sigma);
    if (rc != PRAMAAN_OK) raise_status(rc);
}

}  // namespace gpu
}  // namespace pramaan
