// batch.cuh — many LPs solved together by the adaptive restarted PDHG.
//
// The K LPs of a batch are packed into one block-diagonal LP (rows, columns
// and non-zeros concatenated), so every half-iteration of every LP is ONE
// launch of the tiled product over the packed operand: the tile schedule
// splits the packed non-zeros evenly over the GPU, whatever the sizes of the
// individual LPs, and the whole check interval is one CUDA graph.  Per-LP
// state lives in small device arrays indexed by each row's / column's LP:
//   * the steps are stored already multiplied by the LP's eta * omega (dual)
//     and eta / omega (primal); an omega update rescales that LP's segment,
//     and a converged LP is frozen by zero steps (its iterate no longer
//     moves, so the fused epilogues need no per-LP branch);
//   * relative-KKT sums, movement norms and the reference residuals are
//     per-element contributions reduced per LP in a fixed order (chunks of
//     4096 elements that never straddle two LPs, then the LP's chunks in
//     order), so a batch is deterministic run to run;
//   * restarts, omega updates and the FP64 refinement folds act on the LPs
//     that asked for them (an action code per LP);
//   * when the LPs still iterating hold less than half (Halpern mode: three
//     quarters) of the operand's non-zeros, the operand is rebuilt from them alone and every per-row /
//     per-column array is gathered into the new layout (converged LPs leave
//     their answers in full-layout output arrays first), so the cost of an
//     iteration follows the work that is left.
// Each LP follows exactly the single-LP adaptive method (pdhg_adaptive.cu):
// Ruiz + Pock-Chambolle steps, its own step size eta_k from a per-LP power
// iteration, its own primal weight, averages, KKT restarts and FP64 master
// iterates with FP32 corrections.
#pragma once

#include <vector>

#include "csr_device.cuh"
#include "epilogues.cuh"

namespace pb {

class AdaptiveBatch {
public:
    // `warm` (may be NULL) gives LP k's starting point warm[k]; NULL members
    // keep the cold start for that part.
    AdaptiveBatch(const pramaan_lp* lps, int count, const pramaan_pdhg_options& opt,
                  const pramaan_warm_start* warm = nullptr);
    ~AdaptiveBatch();
    AdaptiveBatch(const AdaptiveBatch&) = delete;
    AdaptiveBatch& operator=(const AdaptiveBatch&) = delete;

    // Solves every LP; results[k] gets LP k's answer (x, y, row_activity
    // copied into its caller-owned buffers when they are not NULL).
    void solve(const pramaan_lp* lps, pramaan_solve_result* results);

    int rows() const { return m_; }
    int cols() const { return n_; }
    int nnz() const { return nnz_; }
    int compactions() const { return compactions_; }

private:
    struct Lp {
        int index = 0;                 // position in the caller's array
        int r0 = 0, r1 = 0, c0 = 0, c1 = 0;      // rows / columns in the current operand
        int or0 = 0, or1 = 0, oc0 = 0, oc1 = 0;  // ... in the original packed layout
        long long nnz = 0;
        double b_norm = 0, c_norm = 0, c32_inf = 1;
        double eta = 1, omega = 1;
        double kkt_restart = 0, kkt_prev = 0;
        int last_restart = 0;
        long long avg_count = 0;
        int status = PRAMAAN_STATUS_ITERATION_LIMIT;
        int iterations = 0, restarts = 0, checks = 0;
        bool active = true;
        // Halpern mode: fixed-point residual at the last restart point and at
        // the previous check (the restart tests compare against them)
        double fpr0 = 0, fpr_prev = 0;
        bool need_fpr0 = true;
        double rel_p = 0, rel_d = 0, rel_gap = 0;
    };
    struct Segments {                  // chunk table of one side (rows or columns)
        int chunks = 0;
        DevBuf<int> begin;             // [chunks + 1] element offsets
        DevBuf<int> lp_first;          // [K + 1] first chunk of each LP
    };
    struct KktSums { double pr2, dr2, dobj, pobj; bool bad; };

    void build_segments(Segments& s, const std::vector<int>& seg_begin);
    // per-LP sums (or maxima) of `width` interleaved contributions per element
    void reduce(const Segments& s, const double* contrib, int width, bool max_op, int out_off);
    void fetch_out();
    void preconditioned_steps();
    void estimate_step_sizes();
    void apply_steps();
    // k iterations starting at global iteration `iter`
    void iterate(int k, int iter);
    // iteration j of an interval of k (Halpern mode writes the fixed-point
    // residual on the first and the last one)
    void iterate_once(int j, int k);
    void kkt(std::vector<KktSums>& cur, std::vector<KktSums>& avg, bool with_average);
    // Halpern mode on small operands: one cooperative kernel per check interval
    bool use_interval_kernel() const;
    void launch_interval(int k);
    // Halpern mode, LPs of at most kClusterAutoMaxNnz non-zeros (or on
    // request): one cluster per LP runs the whole check interval
    // (cluster_interval.cuh).  build_cluster_lps() lists the LPs of the
    // current layout and picks the cluster size.
    bool use_cluster_kernel() const;
    void build_cluster_lps();
    // the long-row lists of the cluster kernel for the LPs `lps` ({r0, r1, c0, c1})
    void build_cluster_long_rows(const std::vector<int4>& lps);
    void launch_cluster(int k);
    void solve_halpern();
    void materialize_average();
    void push_actions();
    void fold(bool first);
    void finish(const pramaan_lp* lps, pramaan_solve_result* results, double solve_ms);
    void check_status();
    // Rebuilds the operand from the LPs still iterating (see above).
    void compact();
    // Launch shapes of the current operands (the products the iteration runs).
    void tune_products();
    // x_out / y_out (original layout) = master + correction of the LPs in the
    // current operand whose keep flag is 0 (all of them when keep is null).
    void scatter_answers(const int* keep);

    int dev_ = 0;
    cudaStream_t st_ = nullptr;
    pramaan_pdhg_options opt_{};
    int count_ = 0;                    // LPs in the caller's array
    int K_ = 0, m_ = 0, n_ = 0, nnz_ = 0;   // LPs on the GPU, packed sizes
    std::vector<Lp> lp_;
    Segments rseg_, cseg_;
    int compactions_ = 0;

    CsrDevice A_, AT_;                 // current operand
    // the original packed LP (host CSR kept for compaction; device copies of
    // what the final evaluation reads, moved aside at the first compaction)
    std::vector<int> h_rp_, h_ci_;
    std::vector<double> h_val_;
    bool compacted_ = false;
    CsrDevice full_A_, full_AT_;
    DevBuf<double> full_cmin64_, full_rlo64_, full_rhi64_, full_vlo64_, full_vhi64_;
    DevBuf<int> full_lp_row_, full_lp_col_;
    Segments full_rseg_, full_cseg_;
    DevBuf<int> row_orig_, col_orig_;  // current -> original index (after a compaction)
    DevBuf<double> x_out_, y_out_;     // answers in the original layout
    int full_m_ = 0, full_n_ = 0;
    DevBuf<int> keep_;
    int* h_keep_ = nullptr;
    DevBuf<int> lp_row_, lp_col_, status_;
    DevBuf<double> cmin64_, rlo64_, rhi64_, vlo64_, vhi64_;
    DevBuf<float> c_, lr_, ur_, lx_, ux_, sig0_, tau0_, sigma_, tau_, x_, xbar_, y_;
    DevBuf<float> xa_, ya_, xl_, yl_, rscale_, cscale_, ones_, ym32_;
    DevBuf<double> xsum_, ysum_, xm64_, ym64_, actm64_, rcm64_;
    DevBuf<double> rcon_, ccon_, chunk_out_, lp_out_;
    DevBuf<int> action_;
    bool halpern_ = false;             // PRAMAAN_ALGO_HALPERN
    DevBuf<int> restart_iter_, iter_base_;   // per LP: iteration of the last restart; the interval's first iteration
    int* h_restart_iter_ = nullptr;
    DevBuf<double> fpr_c_[2], fpr_r_[2];     // fixed-point residual terms, first / last iteration of an interval
    DevBuf<unsigned> gsync_;                 // grid barrier of the interval kernel {count, generation}
    bool cluster_ok_ = false;                // flat operands kept, cluster kernel allowed
    bool cluster_auto_ = false;              // every LP small enough for the automatic choice
    int cluster_nlps_ = 0, cluster_size_ = 1;
    DevBuf<int4> cluster_lps_;               // {r0, r1, c0, c1} per LP of the current layout
    // rows of A and of A^T longer than kClusterLongRow, per LP of the current
    // layout (ranges {a0, a1, at0, at1} into the two lists)
    DevBuf<int4> cluster_long_range_;
    DevBuf<int> cluster_long_a_, cluster_long_at_;
    DevBuf<double> xw_, yw_;           // warm start (original layout), empty when cold
    DevBuf<double> inv_;
    DevBuf<float> dscale_, pscale_, lp_f_;
    // pinned host mirrors of the per-LP arrays
    int* h_action_ = nullptr;
    double* h_inv_ = nullptr;
    float* h_dscale_ = nullptr;
    float* h_pscale_ = nullptr;
    float* h_lp_f_ = nullptr;
    double* h_out_ = nullptr;          // [K * kOutWidth]
    int* h_status_ = nullptr;

    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t graph_exec_ = nullptr;
    int graph_iters_ = 0;
};

}  // namespace pb
