// cuda_backend.hpp — a pramaan::Backend (include/pramaan/gpu/backend.hpp:36-57)
// that solves LP relaxations on the GPU with libpramaan_b200: the "CudaBackend"
// the reference's backend header lists as future work.  Compiled inside a
// PRAMAAN tree; the header itself needs no CUDA types.
#pragma once

#include <memory>

#include "pramaan/gpu/backend.hpp"

namespace pramaan {
namespace gpu {

struct CudaBackendOptions {
    // Relative KKT tolerance of the GPU solve (the FP64-refined restarted
    // Halpern PDHG); RevisedSimplex::Options::tolerance is a pivoting
    // tolerance, not a solution accuracy, so it is not used for this.
    double tolerance = 1e-8;
    int max_iterations = 1000000;
    int device = 0;
};

// The GPU backend.  solve_lp_relaxation returns the SolveResult of the GPU
// solve (x, objective, row activity, residuals by the reference criterion);
// status kOptimal means the relative KKT error met `tolerance`.  Concurrent
// calls are safe: every solve owns its stream and device memory.
std::unique_ptr<Backend> make_cuda_backend(const CudaBackendOptions& options = CudaBackendOptions());

}  // namespace gpu
}  // namespace pramaan
