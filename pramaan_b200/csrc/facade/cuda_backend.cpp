// cuda_backend.cpp — see cuda_backend.hpp.
#include "cuda_backend.hpp"

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "pramaan_b200.h"

namespace pramaan {
namespace gpu {
namespace {

class CudaBackend final : public Backend {
public:
    explicit CudaBackend(const CudaBackendOptions& o) : opt_(o) {}

    SolveResult solve_lp_relaxation(const ModelIR& model, const RevisedSimplex::Options&) override {
        const int m = static_cast<int>(model.numRows());
        const int n = static_cast<int>(model.numVars());
        // the CSR of the model, values as FP64 (integer variable types are ignored:
        // this is the continuous relaxation)
        const auto& A = model.A;
        static const int32_t kZero = 0;
        const int32_t* rp = A.rowPtr().empty() ? &kZero : A.rowPtr().data();
        pramaan_lp lp{};
        lp.num_rows = m;
        lp.num_cols = n;
        lp.nnz = static_cast<int32_t>(A.nnz());
        lp.obj_sense = model.obj_sense == ObjSense::kMaximize ? PRAMAAN_MAXIMIZE : PRAMAAN_MINIMIZE;
        lp.obj_offset = model.obj_offset;
        lp.obj_coeffs = model.obj_coeffs.data();
        lp.row_ptr = rp;
        lp.col_idx = A.colIdx().data();
        lp.values = A.values().data();
        lp.row_lower = model.row_lower.data();
        lp.row_upper = model.row_upper.data();
        lp.var_lower = model.var_lower.data();
        lp.var_upper = model.var_upper.data();
        pramaan_pdhg_options o;
        pramaan_pdhg_default_options(&o);
        o.algorithm = PRAMAAN_ALGO_HALPERN;
        o.termination = PRAMAAN_TERM_RELATIVE_KKT;
        o.refine = 1;
        o.tolerance = opt_.tolerance;
        o.max_iterations = opt_.max_iterations;
        o.check_frequency = 64;
        o.device = opt_.device;
        SolveResult result;
        result.x.assign(static_cast<size_t>(n), 0.0);
        result.row_activity.assign(static_cast<size_t>(m), 0.0);
        std::vector<double> y(static_cast<size_t>(m), 0.0);
        pramaan_solve_result r{};
        r.x = n ? result.x.data() : nullptr;
        r.row_activity = m ? result.row_activity.data() : nullptr;
        r.y = m ? y.data() : nullptr;
        const int rc = pramaan_pdhg_solve(&lp, &o, &r);
        if (rc != PRAMAAN_OK) {
            const std::string msg = pramaan_last_error();
            if (rc == PRAMAAN_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
            throw std::runtime_error(msg);
        }
        result.status = static_cast<SolveStatus>(r.status);
        result.iterations = r.iterations;
        result.objective_value = r.objective_value;
        result.primal_residual = r.primal_residual;
        result.dual_residual = r.dual_residual;
        return result;
    }

private:
    CudaBackendOptions opt_;
};

}  // namespace

std::unique_ptr<Backend> make_cuda_backend(const CudaBackendOptions& options) {
    return std::make_unique<CudaBackend>(options);
}

}  // namespace gpu
}  // namespace pramaan
