// pdhg_engine.cuh — device-resident PDHG state and the host driver loop.
#pragma once

#include <vector>

#include "csr_device.cuh"
#include "epilogues.cuh"
#include "panel.cuh"

namespace pb {

// Makes `dev` current for the lifetime of the guard and restores the
// caller's device afterwards.
class DeviceGuard {
public:
    explicit DeviceGuard(int dev) {
        PB_CUDA_CHECK(cudaGetDevice(&prev_));
        if (dev != prev_) PB_CUDA_CHECK(cudaSetDevice(dev));
    }
    ~DeviceGuard() { cudaSetDevice(prev_); }

private:
    int prev_ = 0;
};

void validate_lp(const pramaan_lp& lp);
void validate_options(const pramaan_pdhg_options& opt);

class PdhgEngine {
public:
    PdhgEngine(const pramaan_lp& lp, const pramaan_pdhg_options& opt);
    ~PdhgEngine();
    PdhgEngine(const PdhgEngine&) = delete;
    PdhgEngine& operator=(const PdhgEngine&) = delete;

    int device() const { return dev_; }
    cudaStream_t stream() const { return st_; }
    int rows() const { return m_; }
    int cols() const { return n_; }

    // `k` reference iterations, asynchronous.
    void iterate(int k);
    // Reference FP64 residuals of the current iterate (synchronises).
    void residuals(double& pv, double& dv, bool& nonfinite);
    // Reference restart: y <- 0, x̄ <- x.
    void restart();
    void get_iterates(float* h_x, float* h_y);
    // Full solve loop (src/gpu/pdhg_solver.cu:319-410 semantics).
    void solve(const pramaan_lp& lp, pramaan_solve_result* res);

    void kernel_times(double* ms_dual, double* ms_primal, long long* launches, bool reset);
    double bytes_dual() const;
    double bytes_primal() const;
    int hot_slots_dual() const { return A_.hot; }
    // the tiled primal product's operand: the remaining entries when Aᵀy is split
    int hot_slots_primal() const { return panel_t_.active ? panel_t_.rest.hot : AT_.hot; }
    // the tiled dual product's operand: the short rows when A x̄ is split over panels
    int gather_l1_dual() const { return panel_.active ? panel_.S.gather_l1 : A_.gather_l1; }
    int gather_l1_primal() const { return panel_t_.active ? panel_t_.rest.gather_l1 : AT_.gather_l1; }
    int blocks_dual() const { return panel_.active ? panel_.S.tuned_blocks_per_sm : A_.tuned_blocks_per_sm; }
    // Column-panel split of the A x̄ product (reference mode): panels, long rows
    // and their non-zeros, the row length from which a row is long (0: not split).
    // The hot part of Aᵀy: the rows of A whose y every block holds, their
    // non-zeros (0: the tiled product alone).
    void panel_info(int* panels, int* long_rows, long long* long_nnz, int* min_len, int* hot_rows,
                    long long* hot_nnz) const {
        *panels = panel_.active ? panel_.panels : 0;
        *long_rows = panel_.active ? panel_.long_rows : 0;
        *long_nnz = panel_.active ? panel_.long_nnz : 0;
        *min_len = panel_.active ? panel_.min_len : 0;
        *hot_rows = panel_t_.active ? panel_t_.hot_rows : 0;
        *hot_nnz = panel_t_.active ? panel_t_.hot_nnz : 0;
    }
    int blocks_primal() const { return panel_t_.active ? panel_t_.rest.tuned_blocks_per_sm : AT_.tuned_blocks_per_sm; }
    void synchronize();

    // ---- adaptive mode (pdhg_adaptive.cu) ----
    struct Kkt {
        double rel_p = 0, rel_d = 0, rel_gap = 0;   // PDLP relative KKT components
        double pr2 = 0, dr2 = 0, pobj = 0, dobj = 0;  // raw sums
        bool nonfinite = false;
        double weighted(double omega) const;          // restart metric
        bool converged(double tol) const { return rel_p <= tol && rel_d <= tol && rel_gap <= tol; }
    };
    // Relative KKT (FP64, original problem) of the current iterate and of the
    // epoch's average, both as master + correction (synchronises).
    void kkt_pair(Kkt& cur, Kkt& avg);
    double primal_weight() const { return omega_; }
    double step_size() const { return eta_; }

private:
    void iterate_once();
    void launch_dual();
    void launch_primal();
    void check_device_status();
    void build_graph(int k);
    void drain_events();
    // adaptive mode
    void setup_adaptive(const pramaan_lp& lp);
    void preconditioned_steps();
    double estimate_operator_norm();
    void set_weight(double omega);
    void materialize_average();
    void restart_to(bool average);
    // Folds the correction (d, e) into the FP64 master (x_m, y_m) — or, with
    // `first`, sets the master to the starting point — and refreshes the FP32
    // vectors the correction iteration reads; d = e = d̄ = 0 afterwards.
    void fold(bool first);
    // x64_ = x_m + d, y64_ = y_m + e; the FP32 vectors back to the original LP.
    void finish_adaptive();
    void solve_adaptive(pramaan_solve_result* res);
    double dist2(const float* a, const float* b, const float* scale, int len);
    void reference_residuals64(double& pv, double& dv, bool& nonfinite);

    int dev_ = 0;
    cudaStream_t st_ = nullptr;
    pramaan_pdhg_options opt_{};
    int m_ = 0, n_ = 0;
    double c_norm_ = 1.0;
    bool adaptive_ = false;

    CsrDevice A_, AT_;
    PanelSplit panel_;   // A x̄ over column panels (reference mode, power-law operands)
    PanelHot panel_t_;   // the longest rows' part of Aᵀy over the same panels
    DevBuf<float> c_, lr_, ur_, lx_, ux_, sigma_, tau_, x_, y_, xbar_;
    DevBuf<double> rlo64_, rhi64_, vlo64_, vhi64_, slots_;
    DevBuf<int> status_;
    double* h_slots_ = nullptr;   // pinned
    int* h_status_ = nullptr;     // pinned

    // adaptive-mode state.  The FP32 iterate buffers hold the correction
    // (x_ = d, y_ = e, xbar_ = d̄) and the FP32 problem vectors its folded data
    // (c_ = c + A^T y_m, lr_/ur_ = A x_m - l_r / - u_r, lx_/ux_ = bounds - x_m).
    DevBuf<double> cmin64_, xsum_, ysum_, part_, red_;
    DevBuf<float> rscale_, cscale_, xa_, ya_, xl_, yl_, scal_;
    DevBuf<double> xm64_, ym64_, actm64_, rcm64_;   // FP64 master, A x_m, c + A^T y_m
    DevBuf<float> ym32_;
    double* h_red_ = nullptr;     // pinned, kPartSlots
    double eta_ = 1.0, omega_ = 1.0;
    double b_norm_ = 0.0, c_norm2_ = 0.0;
    long long avg_count_ = 0;
    int folds_ = 0;
    // FP64 answer of an adaptive solve (x_m + d, y_m + e)
    bool master_out_ = false;
    DevBuf<double> x64_, y64_;

    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    int graph_iters_ = 0;

    // kernel timing (profile_kernels)
    struct EvPair { cudaEvent_t a, b; int kind; };
    std::vector<EvPair> ev_pool_;
    size_t ev_used_ = 0;
    double ms_dual_ = 0.0, ms_primal_ = 0.0;
    long long launches_ = 0;
};

}  // namespace pb
