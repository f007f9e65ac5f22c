// check_cuda_backend.cpp — the GPU Backend (pramaan_b200/csrc/facade/cuda_backend.hpp)
// against the reference's CPU Backend (make_cpu_backend, src/gpu/backend_cpu.cpp)
// on the reference's afiro fixture and two small LPs built through the
// reference's ModelIR.  Prints "CUDA BACKEND CHECK PASSED" on success.
#include <cmath>
#include <cstdio>
#include <memory>
#include <vector>

#include "cuda_backend.hpp"
#include "pramaan/gpu/backend.hpp"
#include "pramaan/ir.hpp"
#include "pramaan/mps_parser.hpp"

using namespace pramaan;

static int failures = 0;

static void compare(const char* name, const ModelIR& model) {
    auto cpu = make_cpu_backend();
    gpu::CudaBackendOptions go;
    go.tolerance = 1e-9;
    auto gpu = gpu::make_cuda_backend(go);
    RevisedSimplex::Options so;
    so.max_iterations = 100000;
    const SolveResult a = cpu->solve_lp_relaxation(model, so);
    const SolveResult b = gpu->solve_lp_relaxation(model, so);
    const double tol = 1e-6 * (1.0 + std::fabs(a.objective_value));
    const bool ok = a.status == SolveStatus::kOptimal && b.status == SolveStatus::kOptimal &&
                    std::fabs(a.objective_value - b.objective_value) <= tol &&
                    static_cast<int>(b.x.size()) == model.numVars() && b.primal_residual <= 1e-6;
    std::printf("%-10s cpu %.10g  gpu %.10g  (%d iterations, primal residual %.2e) %s\n", name, a.objective_value,
                b.objective_value, b.iterations, b.primal_residual, ok ? "ok" : "FAIL");
    if (!ok) ++failures;
}

int main() {
    {   // max 3x + 5y, x <= 4, 2y <= 12, 3x + 2y <= 18 (optimum 36)
        ModelIR m;
        m.obj_sense = ObjSense::kMaximize;
        m.obj_coeffs = {3.0, 5.0};
        m.A = CSRMatrix({0, 1, 2, 4}, {0, 1, 0, 1}, {1.0, 2.0, 3.0, 2.0}, 2);
        m.row_lower = {-kInfinity, -kInfinity, -kInfinity};
        m.row_upper = {4.0, 12.0, 18.0};
        m.var_lower = {0.0, 0.0};
        m.var_upper = {kInfinity, kInfinity};
        m.var_types = {VarType::kContinuous, VarType::kContinuous};
        m.row_names = {"r0", "r1", "r2"};
        m.var_names = {"x", "y"};
        compare("wyndor", m);
    }
    {   // min x + 2y + 3z, x + y + z = 5, x - y >= -1, 0 <= x,y,z <= 4
        ModelIR m;
        m.obj_sense = ObjSense::kMinimize;
        m.obj_coeffs = {1.0, 2.0, 3.0};
        m.A = CSRMatrix({0, 3, 5}, {0, 1, 2, 0, 1}, {1.0, 1.0, 1.0, 1.0, -1.0}, 3);
        m.row_lower = {5.0, -1.0};
        m.row_upper = {5.0, kInfinity};
        m.var_lower = {0.0, 0.0, 0.0};
        m.var_upper = {4.0, 4.0, 4.0};
        m.var_types = {VarType::kContinuous, VarType::kContinuous, VarType::kContinuous};
        m.row_names = {"r0", "r1"};
        m.var_names = {"x", "y", "z"};
        compare("equality", m);
    }
    try {
        const ModelIR afiro = parse_mps("tests/data/afiro.mps");
        compare("afiro", afiro);
    } catch (const std::exception& e) {
        std::printf("afiro: %s\n", e.what());
        ++failures;
    }
    std::printf(failures ? "CUDA BACKEND CHECK FAILED\n" : "CUDA BACKEND CHECK PASSED\n");
    return failures ? 1 : 0;
}
