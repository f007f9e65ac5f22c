/*
 * pramaan_b200.h — C ABI of libpramaan_b200.so, the sm_100a restarted-PDHG LP
 * solver that stands in for PRAMAAN's GPU PDHG path (src/gpu/).
 *
 * Every entry point is extern "C", takes plain pointers and sizes, and
 * returns an int status (PRAMAAN_OK or a negative PRAMAAN_ERR_*).  The text of
 * the last failure on the calling thread is available from
 * pramaan_last_error(); for CUDA failures it has the reference's form
 * "CUDA error in <file>:<line> - <message>" (src/gpu/cuda_utils.cuh:8-15).
 * Solver outcomes (optimal, iteration limit, numerical failure) are reported
 * through pramaan_solve_result.status and are never errors.
 *
 * Data types follow the reference's ModelIR (include/pramaan/ir.hpp:62-119)
 * and CSRMatrix (include/pramaan/sparse_matrix.hpp:28-181): int32 indices,
 * FP64 values, ranged rows row_lower <= A x <= row_upper, boxed variables,
 * +-1e30 as "infinite".  All host arrays are owned by the caller, read during
 * the call and never retained.
 */
#ifndef PRAMAAN_B200_H
#define PRAMAAN_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define PRAMAAN_API __attribute__((visibility("default")))
#else
#define PRAMAAN_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes ------------------------------------------------------- */
#define PRAMAAN_OK 0
#define PRAMAAN_ERR_INVALID_ARGUMENT (-1)
#define PRAMAAN_ERR_CUDA (-2)
#define PRAMAAN_ERR_DEVICE_TIMEOUT (-3)
#define PRAMAAN_ERR_INTERNAL (-4)

/* ---- solver status: values of pramaan::SolveStatus
 *      (include/pramaan/simplex.hpp:26-33) ---------------------------------- */
#define PRAMAAN_STATUS_OPTIMAL 0
#define PRAMAAN_STATUS_INFEASIBLE 1
#define PRAMAAN_STATUS_UNBOUNDED 2
#define PRAMAAN_STATUS_ITERATION_LIMIT 3
#define PRAMAAN_STATUS_NUMERICAL_FAILURE 4
#define PRAMAAN_STATUS_WARM_START_REJECTED 5

/* ---- objective sense (pramaan::ObjSense, include/pramaan/ir.hpp:28-31) --- */
#define PRAMAAN_MINIMIZE 0
#define PRAMAAN_MAXIMIZE 1

/* ---- algorithm / termination selectors (extensions) --------------------- */
#define PRAMAAN_ALGO_REFERENCE 0 /* the reference iteration, step sizes and restart rule */
#define PRAMAAN_ALGO_ADAPTIVE 1  /* same iteration with Ruiz + Pock-Chambolle steps, primal
                                    weight, averaging and KKT-based adaptive restarts;
                                    needs PRAMAAN_TERM_RELATIVE_KKT */
#define PRAMAAN_ALGO_HALPERN 2   /* restarted Halpern PDHG with reflection: the same
                                    preconditioned steps and primal weight, each
                                    iterate moved to w((1+r)T(z) - r z) + (1-w) z0
                                    (w = (k+1)/(k+2), r = 1, z0 the restart point),
                                    restarts on the fixed-point residual; needs
                                    PRAMAAN_TERM_RELATIVE_KKT and refine = 1 */
#define PRAMAAN_TERM_REFERENCE 0 /* abs. max primal violation, rel. max dual violation */
#define PRAMAAN_TERM_RELATIVE_KKT 1 /* relative primal, dual residual and gap (L2, FP64) */

/* LP in the reference's ModelIR form. */
typedef struct pramaan_lp {
    int32_t num_rows;          /* m                                            */
    int32_t num_cols;          /* n                                            */
    int32_t nnz;               /* row_ptr[m]                                   */
    int32_t obj_sense;         /* PRAMAAN_MINIMIZE / PRAMAAN_MAXIMIZE          */
    double obj_offset;         /* constant added to c^T x for reporting        */
    const double* obj_coeffs;  /* [n]                                          */
    const int32_t* row_ptr;    /* [m + 1]                                      */
    const int32_t* col_idx;    /* [nnz]                                        */
    const double* values;      /* [nnz]                                        */
    const double* row_lower;   /* [m]                                          */
    const double* row_upper;   /* [m]                                          */
    const double* var_lower;   /* [n]                                          */
    const double* var_upper;   /* [n]                                          */
} pramaan_lp;

/* Options.  The first three fields are pramaan::gpu::PdhgOptions
 * (include/pramaan/gpu/pdhg_solver.hpp:9-13) with the same defaults; the rest
 * are extensions whose defaults reproduce the reference behaviour. */
typedef struct pramaan_pdhg_options {
    double tolerance;         /* 1e-6                                          */
    int32_t max_iterations;   /* 100000                                        */
    int32_t check_frequency;  /* 100 (must be >= 1)                            */
    int32_t algorithm;        /* PRAMAAN_ALGO_REFERENCE                        */
    int32_t termination;      /* PRAMAAN_TERM_REFERENCE                        */
    int32_t device;           /* CUDA device ordinal, default 0                */
    int32_t use_graph;        /* 1: replay each check interval as a CUDA graph */
    int32_t profile_kernels;  /* 1: time every product kernel with CUDA events */
    int32_t refine;           /* adaptive mode, 1 (default): FP64 master iterates
                                 on the device, the FP32 iteration runs on the
                                 correction and is folded into them at every
                                 restart (iterative refinement), so tolerances
                                 to about 1e-10 are reachable; 0: plain FP32
                                 iterates (resolution about 1e-6)               */
    double reserved_d;
    int32_t persistent;       /* Halpern mode, how a check interval runs:
                                 0 (default): one thread-block cluster per LP
                                 runs the whole interval in one launch when
                                 every LP has at most 2^20 non-zeros, else as -1;
                                 2: the cluster kernel for any size;
                                 1: one cooperative kernel over the packed
                                 operand (grid barriers between the products);
                                 -1: the two tiled products per iteration,
                                 captured in a CUDA graph with dependent
                                 launches                                       */
    int32_t gather_cache;     /* 0 (default): the products over a large operand
                                 whose gathers concentrate on few entries (the
                                 transpose of an LP with power-law row lengths)
                                 keep those entries in shared memory, and the
                                 launch autotuner caches the gathers of the
                                 other large operands in L1 where that is
                                 faster (local column patterns); 1: as 0, but
                                 L1-cached gathers on every operand without hot
                                 entries; -1: plain L2 gathers only.  The
                                 results are identical in every mode            */
    int32_t launch_blocks;    /* 0 (default): the launch autotuner picks the
                                 resident blocks per SM of the products over a
                                 large operand; > 0: that many (capped by what
                                 fits), only the gather mode is then timed,
                                 and not even that when gather_cache is 1 or
                                 -1: a fixed launch shape, for reproducible
                                 profiles                                       */
    int32_t panel_split;      /* reference algorithm, the two products:
                                 0 (default): when rows of at least twice the
                                 panel count of entries hold half or more of
                                 A's non-zeros (power-law row lengths, at
                                 least 4 Mi of them), those long rows are
                                 computed over column panels of x̄ held in
                                 shared memory, one per SM, and the other rows
                                 by the tiled product; 1: the same split
                                 whenever it is feasible; >= 2: the split with
                                 rows of at least that many entries as the long
                                 rows; -1: the tiled products only.  With A x̄
                                 split, Aᵀy is split too where it can be: every
                                 SM holds y of the longest rows of A and sums
                                 their entries for its panel's columns, the
                                 tiled product the other entries.  Sums are
                                 deterministic in every mode; a split changes
                                 the order of the additions within a row      */
    int32_t reserved[2];
} pramaan_pdhg_options;

/* Result, mirroring pramaan::SolveResult (include/pramaan/simplex.hpp:40-76).
 * x, row_activity and y are caller-owned output buffers (may be NULL). */
typedef struct pramaan_solve_result {
    int32_t status;            /* PRAMAAN_STATUS_*                              */
    int32_t iterations;        /* = max_iterations when not optimal             */
    double primal_residual;    /* reference criterion, FP64                     */
    double dual_residual;      /* reference criterion, FP64                     */
    double objective_value;    /* c^T x + obj_offset in the model's own sense   */
    double* x;                 /* out [n]                                       */
    double* row_activity;      /* out [m] = A x in FP64                         */
    double* y;                 /* out [m], dual iterate (reference sign)        */
    int32_t restarts;          /* restarts performed                            */
    int32_t checks;            /* convergence checks performed                  */
    double solve_ms;           /* wall time inside the call                     */
    double rel_primal;         /* relative KKT of the result (adaptive mode):   */
    double rel_dual;           /*   ||primal residual||/(1+||b||), ||dual      */
    double rel_gap;            /*   residual||/(1+||c||), |p-d|/(1+|p|+|d|)     */
    double primal_weight;      /* final omega (adaptive mode)                   */
    double step_size;          /* eta (adaptive mode)                           */
    double compactions;        /* batch solves: operand rebuilds during the batch */
} pramaan_solve_result;

/* Library identification. */
PRAMAAN_API const char* pramaan_version(void);
/* Text of the last failure on the calling thread ("" when none). */
PRAMAAN_API const char* pramaan_last_error(void);

/* Fills *opt with the defaults listed above. */
PRAMAAN_API void pramaan_pdhg_default_options(pramaan_pdhg_options* opt);

/* One complete solve: replaces pramaan::gpu::PdhgSolver::solve
 * (src/gpu/pdhg_solver.cu:169-411).  Uploads the LP, runs the PDHG loop on the
 * GPU (FP32 iterates, FP64 residual checks on the device), and writes the
 * result.  Returns PRAMAAN_OK when the solve ran (whatever its status). */
PRAMAAN_API int pramaan_pdhg_solve(const pramaan_lp* lp, const pramaan_pdhg_options* opt,
                       pramaan_solve_result* result);

/* Many LPs solved together (no reference counterpart; the batch client of
 * the reference is PdhgSolver::solve called once per LP, e.g. per
 * branch-and-bound node relaxation or rolling-horizon window).  The LPs are
 * packed into one block-diagonal operand, so each half-iteration of all of
 * them is one kernel launch; each LP keeps its own step size, primal weight,
 * restarts, FP64 refinement and termination, and is frozen once it meets the
 * tolerance.  opt->algorithm must be PRAMAAN_ALGO_ADAPTIVE or
 * PRAMAAN_ALGO_HALPERN with PRAMAAN_TERM_RELATIVE_KKT (NULL: the defaults with
 * PRAMAAN_ALGO_HALPERN and PRAMAAN_TERM_RELATIVE_KKT).
 * results[k] is LP k's result, with caller-owned x / y / row_activity
 * buffers as in pramaan_pdhg_solve; solve_ms is the whole batch's time.
 * LPs without variables or with non-finite costs get the reference's early
 * answers.  The packed sizes must stay below 2^30 rows, columns and
 * non-zeros. */
PRAMAAN_API int pramaan_pdhg_solve_batch(const pramaan_lp* lps, int32_t count,
                                         const pramaan_pdhg_options* opt,
                                         pramaan_solve_result* results);

/* A starting point for one LP (no reference counterpart: the reference's
 * only warm start is the dual simplex basis of BasisState,
 * include/pramaan/dual_simplex.hpp:63-130).  Also used as a training target
 * of the warm-start network. */
typedef struct pramaan_warm_start {
    const double* x;        /* [n] primal point, or NULL: clamp(0, l, u)          */
    const double* y;        /* [m] dual point with the solver's sign (the y of a
                               pramaan_solve_result), or NULL: 0                 */
    double primal_weight;   /* > 0: initial primal weight; otherwise the default  */
} pramaan_warm_start;

/* pramaan_pdhg_solve_batch started from given points: LP k starts from
 * warm[k] (x clamped into its bounds, y as given, omega as given) instead of
 * the cold start.  warm == NULL is pramaan_pdhg_solve_batch.  The iteration,
 * restarts and termination are unchanged, so a result is judged exactly as a
 * cold one. */
PRAMAAN_API int pramaan_pdhg_solve_batch_warm(const pramaan_lp* lps, int32_t count,
                                              const pramaan_pdhg_options* opt,
                                              const pramaan_warm_start* warm,
                                              pramaan_solve_result* results);

/* ---- precision ladder ---------------------------------------------------------
 * The two-rung controller of pramaan::PrecisionLadder
 * (src/gpu/precision_ladder.cpp:55-181) with a GPU FP64 rung between them:
 *   rung 1  the reference FP32 PDHG (as PdhgSolver::solve, gpu_* options);
 *           accepted iff status optimal and both reference residuals (the
 *           solver's FP64 ComputeFp64Residuals check) are <= residual_threshold
 *           — exactly the reference's gate;
 *   rung 2  (refine != 0) the adaptive PDHG with FP64 iterative refinement on
 *           the GPU to refine_tolerance relative KKT; accepted by the same
 *           gate on its own reference residuals;
 *   rung 3  escalation: the caller's CPU FP64 solver (the reference runs
 *           RevisedSimplex with the GPU x as primal_start_hint); result->x then
 *           holds that hint (the better GPU point).
 * With refine == 0 the decisions are the reference's. */
#define PRAMAAN_LADDER_GPU_FP32 0
#define PRAMAAN_LADDER_GPU_FP64_REFINED 1
#define PRAMAAN_LADDER_ESCALATE 2
/* values of PrecisionLadderResult::EscalationReason (include/pramaan/gpu/precision_ladder.hpp) */
#define PRAMAAN_ESCALATION_NONE 0
#define PRAMAAN_ESCALATION_HIGH_PRIMAL_RESIDUAL 1
#define PRAMAAN_ESCALATION_HIGH_DUAL_RESIDUAL 2
#define PRAMAAN_ESCALATION_GPU_ITERATION_LIMIT 3
#define PRAMAAN_ESCALATION_GPU_NUMERICAL_FAILURE 4
#define PRAMAAN_ESCALATION_GPU_NOT_OPTIMAL 5

typedef struct pramaan_ladder_options {
    double residual_threshold;       /* T, 1e-6 (Options::residual_threshold)      */
    int32_t gpu_max_iterations;      /* 100000                                     */
    int32_t gpu_check_frequency;     /* 100                                        */
    double gpu_tolerance;            /* 1e-6                                       */
    int32_t refine;                  /* 1: run rung 2 before escalating            */
    int32_t refine_max_iterations;   /* 400000                                     */
    double refine_tolerance;         /* 1e-9 relative KKT                          */
    int32_t device;                  /* 0                                          */
    int32_t reserved[3];
} pramaan_ladder_options;

typedef struct pramaan_ladder_result {
    int32_t stage;                   /* PRAMAAN_LADDER_*                           */
    int32_t escalation_reason;       /* rung 1's reason (PRAMAAN_ESCALATION_*)      */
    int32_t refine_escalation_reason;/* rung 2's reason when it ran                */
    int32_t gpu_status, gpu_iterations;
    int32_t refine_status, refine_iterations;
    int32_t reserved;
    double gpu_primal_residual, gpu_dual_residual, gpu_objective, gpu_elapsed_ms;
    double refine_primal_residual, refine_dual_residual, refine_objective, refine_elapsed_ms;
    double rel_primal, rel_dual, rel_gap;   /* relative KKT of the returned point  */
    double objective_value;          /* of the returned point, model's sense       */
    double total_elapsed_ms;
    double* x;                       /* out [n]: the accepted point / CPU hint      */
    double* y;                       /* out [m] (may be NULL)                      */
    double* row_activity;            /* out [m] (may be NULL)                      */
} pramaan_ladder_result;

PRAMAAN_API void pramaan_ladder_default_options(pramaan_ladder_options* opt);
PRAMAAN_API int pramaan_ladder_solve(const pramaan_lp* lp, const pramaan_ladder_options* opt,
                                     pramaan_ladder_result* result);

/* ---- certificates -----------------------------------------------------------
 * FP64 certificate of a point (x, y) of an LP, computed on the GPU.  The first
 * three fields are the reference certificate's (pramaan::generate_certificate,
 * src/certificate/certificate.cpp:23-107: objective, maximum row violation,
 * maximum variable-bound violation; integrality is 0 for LPs); the rest add
 * the dual side the reference leaves empty (std::nullopt there): the relative
 * KKT error of (x, y) in FP64 with the problem in minimisation form and y the
 * solver's dual (the negated multiplier). */
typedef struct pramaan_certificate {
    double objective_value;    /* c^T x + obj_offset in the model's sense       */
    double primal_residual;    /* max over rows of max(l_r - Ax, Ax - u_r, 0)    */
    double bound_violation;    /* max over columns of max(l_x - x, x - u_x, 0)   */
    double rel_primal;         /* ||(dist(Ax,[l_r,u_r]), dist(x,[l_x,u_x]))||_2
                                  / (1 + ||finite row bounds||_2)               */
    double rel_dual;           /* ||rc - proj(rc)||_2 / (1 + ||c||_2), rc = c + A^T y */
    double rel_gap;            /* |p - d| / (1 + |p| + |d|)                      */
    double primal_objective;   /* p = c^T x (minimisation form)                  */
    double dual_objective;     /* d (minimisation form)                          */
    double kkt;                /* max(rel_primal, rel_dual, rel_gap)             */
} pramaan_certificate;

/* Certificates of num_points points of each of `count` LPs: points[p * count
 * + k] is point p of LP k (x NULL: the solver's cold start clamp(0, l, u);
 * y NULL: 0) and its certificate goes to out[p * count + k].  The LPs are
 * packed once for all points. */
PRAMAAN_API int pramaan_certify_batch(const pramaan_lp* lps, int32_t count, const pramaan_warm_start* points,
                                      int32_t num_points, int32_t device, pramaan_certificate* out);

/* ---- learned warm start (no reference counterpart) ------------------------
 * A bipartite constraint-variable graph network (3 message-passing layers,
 * hidden width 64, BF16 weights and activations, FP32 accumulation on the
 * tensor cores) that predicts x, y and the primal weight of each LP of a
 * batch, optionally refining a caller-given hint.  Its parameters are a flat FP32 vector of pramaan_gnn_num_params()
 * entries (the master copy; the forward pass uses them rounded to BF16).   */
typedef struct pramaan_gnn pramaan_gnn;
typedef struct pramaan_gnn_graph pramaan_gnn_graph;

PRAMAAN_API int32_t pramaan_gnn_num_params(void);
/* A network with seeded He-uniform weights on `device`. */
PRAMAAN_API int pramaan_gnn_create(int32_t device, uint64_t seed, pramaan_gnn** out);
PRAMAAN_API int pramaan_gnn_destroy(pramaan_gnn* net);
PRAMAAN_API int pramaan_gnn_get_params(const pramaan_gnn* net, float* params);
/* Replaces the parameters and resets the optimiser state. */
PRAMAAN_API int pramaan_gnn_set_params(pramaan_gnn* net, const float* params);
/* Packs `count` LPs into a device-resident graph (features, both CSR
 * orientations).  `hints` (NULL: none) gives each LP an optional prior guess
 * of its solution (x and / or y, NULL members allowed; the primal weight is
 * ignored) — for a rolling-horizon stream, the previous window's solution
 * shifted by one period; the network reads it as node features and predicts
 * a correction to it.  `targets` (NULL for prediction only) gives each LP's
 * solved point: x [n], y [m] and a positive primal weight.  LPs without
 * variables are skipped (they get no prediction). */
PRAMAAN_API int pramaan_gnn_graph_create(const pramaan_lp* lps, int32_t count,
                                         const pramaan_warm_start* hints,
                                         const pramaan_warm_start* targets, int32_t device,
                                         pramaan_gnn_graph** out);
PRAMAAN_API int pramaan_gnn_graph_destroy(pramaan_gnn_graph* g);
/* Forward pass; writes LP k's predicted x into x_out[k] ([n], may be NULL),
 * y into y_out[k] ([m], may be NULL) and its primal weight into omega_out[k]
 * (x_out, y_out, omega_out may themselves be NULL). */
PRAMAAN_API int pramaan_gnn_predict(pramaan_gnn* net, const pramaan_gnn_graph* g, double* const* x_out,
                                    double* const* y_out, double* omega_out);
/* Forward + backward without an update: *loss and the gradient of the loss
 * with respect to every parameter (grad [pramaan_gnn_num_params()], may be
 * NULL).  The graph must have targets. */
PRAMAAN_API int pramaan_gnn_gradients(pramaan_gnn* net, const pramaan_gnn_graph* g, float* grad,
                                      double* loss);
/* One Adam step (beta 0.9 / 0.999, eps 1e-8) on the loss of graph g; *loss
 * receives the loss before the step. */
PRAMAAN_API int pramaan_gnn_train_step(pramaan_gnn* net, const pramaan_gnn_graph* g, float learning_rate,
                                       double* loss);
/* Number of floats written by pramaan_gnn_forward_trace for graph g. */
PRAMAAN_API int64_t pramaan_gnn_trace_size(const pramaan_gnn_graph* g);
/* Forward pass and a copy of every stored activation as FP32, in order:
 * X_c of layers 1-3 ([m][128] each: h_c input | aggregated h_v), X_v of
 * layers 1-3 ([n][128]), h_c and h_v after layer 3 ([m][64], [n][64]),
 * xhat [n], yhat [m], pooled [K][128], rho [K]  (rows in packed order: LP
 * after LP, LPs without variables left out). */
PRAMAAN_API int pramaan_gnn_forward_trace(pramaan_gnn* net, const pramaan_gnn_graph* g, float* out);

/* ---- test-harness launchers (src/gpu/pdhg.cu:77-241) --------------------- */

/* y_out[m] = A x for the FP32 CSR (row_ptr[m+1], col_idx[nnz], values[nnz]),
 * x[n].  Replaces launch_spmv (src/gpu/pdhg.cu:156-196).  m == 0 writes
 * nothing. */
PRAMAAN_API int pramaan_launch_spmv(const int32_t* row_ptr, const int32_t* col_idx, const float* values,
                        int32_t nnz, const float* x, float* y_out, int32_t m, int32_t n);

/* y_out[n] = A^T x for the same CSR, x[m].  Replaces launch_spmv_t
 * (src/gpu/pdhg.cu:198-241); computed by a gather over a stored transpose
 * (deterministic) instead of an atomic scatter.  m == 0 writes zeros. */
PRAMAAN_API int pramaan_launch_spmv_t(const int32_t* row_ptr, const int32_t* col_idx, const float* values,
                          int32_t nnz, const float* x, float* y_out, int32_t m, int32_t n);

/* One Step-1 dense iteration, in place (src/gpu/pdhg.cu:77-146):
 *   x <- max(0, x - tau * gradient)          (n entries)
 *   y <- y + sigma * (Ax_bar - b)            (m entries) */
PRAMAAN_API int pramaan_launch_pdhg_iteration(float* h_x, float* h_y, const float* h_gradient,
                                  const float* h_Ax_bar, const float* h_b, int32_t n, int32_t m,
                                  float tau, float sigma);

/* y[m] = A x for a CSR that already lives in device memory, allocating
 * nothing.  This entry point has no counterpart in the reference.  It exists
 * for callers that cannot call cudaMalloc where they need the product: drivers
 * that size all device memory up front under a fixed budget (branch-and-bound,
 * rolling-horizon loops), code running while a stream is captured into a CUDA
 * graph, and hosts that own the device memory pool.  All pointers are device
 * pointers owned by the caller (row_ptr[m+1], col_idx[nnz], values[nnz], x[n],
 * y[m]); the work is queued on `stream` (a cudaStream_t, NULL for the legacy
 * default stream) and the call returns without waiting.  Partial sums of rows
 * that cross 2048-entry tiles go to a 512 KiB scratch array compiled into the
 * library (a file-scope __device__ array, held by every GPU that loads the
 * library until exit), which limits nnz to 134,217,728; larger inputs are
 * rejected with PRAMAAN_ERR_INVALID_ARGUMENT.  Every call shares that array:
 * calls on one stream are ordered, calls that overlap on the GPU race.  The
 * first call on a device looks up the array's device address and caches it
 * for that device's primary context; it allocates nothing itself, but under
 * lazy module loading it is where the library's module, and with it the
 * array's storage, may be loaded onto the device.  So make one call per device
 * before capturing a stream or fixing a memory budget.  The CSR must be well
 * formed (row_ptr nondecreasing, row_ptr[0] = 0, row_ptr[m] = nnz); it is not
 * validated, but out-of-range column indices are clamped so they never read
 * outside x, and row_ptr is never read outside [0, m]. */
PRAMAAN_API int pramaan_spmv_noalloc(const int32_t* d_row_ptr, const int32_t* d_col_idx,
                                     const float* d_values, int32_t m, int32_t n, int32_t nnz,
                                     const float* d_x, float* d_y, void* stream);

/* ---- device-resident session (benchmarks and advanced callers) ----------- */

typedef struct pramaan_pdhg_session pramaan_pdhg_session;

/* Uploads the LP and prepares the reference iteration (step sizes, transpose,
 * x0).  opt->algorithm must be PRAMAAN_ALGO_REFERENCE. */
PRAMAAN_API int pramaan_session_create(const pramaan_lp* lp, const pramaan_pdhg_options* opt,
                           pramaan_pdhg_session** out);
PRAMAAN_API int pramaan_session_destroy(pramaan_pdhg_session* s);
/* Runs `iterations` PDHG iterations without convergence checks (asynchronous
 * on the session stream; graph replay when use_graph is set). */
PRAMAAN_API int pramaan_session_iterate(pramaan_pdhg_session* s, int32_t iterations);
/* Waits for the session stream. */
PRAMAAN_API int pramaan_session_synchronize(pramaan_pdhg_session* s);
/* Reference FP64 residuals of the current iterate (synchronises). */
PRAMAAN_API int pramaan_session_residuals(pramaan_pdhg_session* s, double* primal, double* dual);
/* Copies the current FP32 iterates to host buffers (either may be NULL). */
PRAMAAN_API int pramaan_session_get_iterates(pramaan_pdhg_session* s, float* x, float* y);
/* The cudaStream_t the session launches on. */
PRAMAAN_API void* pramaan_session_stream(pramaan_pdhg_session* s);
/* Accumulated CUDA-event time (ms) of the two products and the number of
 * kernels they launched since the last reset (a product is its main kernel
 * plus, when rows cross tiles, their completion kernel; profile_kernels must
 * be set; synchronises). */
PRAMAAN_API int pramaan_session_kernel_times(pramaan_pdhg_session* s, double* ms_dual, double* ms_primal,
                                 int64_t* launches, int32_t reset);
/* Algorithmic bytes of one launch of each product kernel (see the layout
 * notes in the library documentation). */
PRAMAAN_API int pramaan_session_kernel_bytes(pramaan_pdhg_session* s, double* bytes_dual,
                                 double* bytes_primal);
/* Frees the device memory the library keeps for reuse on device `device`
 * (-1: every device).  Solves allocate their operands and temporaries from a
 * per-device cache (at most 32 GB kept per device) so that repeated solves
 * skip cudaMalloc / cudaFree; this returns that memory to the driver. */
PRAMAAN_API int pramaan_release_cached_memory(int32_t device);

/* Measures the current device's random-gather rate: 4-byte loads of d_x[0, n)
 * (a device array) at hashed uniform indices, 16 in flight per thread, 8
 * blocks of 256 threads per SM, nothing else read or written; L1-cached loads
 * when `cached` is set, else ld.global.cg.  Writes the median over `reps`
 * timed launches in gathers per second.  The call runs on a stream of its own
 * and does not wait for other streams: d_x must be ready.  No reference counterpart: it is the
 * ceiling the benchmark reports the products against, since on a random
 * sparsity pattern every non-zero costs one such gather. */
PRAMAAN_API int pramaan_measure_gather_rate(const float* d_x, int32_t n, int32_t cached, int32_t reps,
                                            double* gathers_per_s);

/* Gather modes (option gather_cache) of the dual product's operand A and the
 * primal product's operand A^T: hot gather slots (entries of x kept in shared
 * memory), whether the gathers are cached in L1 (1) or not (0), and the
 * resident blocks per SM the launch autotuner chose (0: the default grid).
 * Any pointer may be NULL. */
PRAMAAN_API int pramaan_session_gather_info(pramaan_pdhg_session* s, int32_t* slots_dual,
                                int32_t* slots_primal, int32_t* l1_dual, int32_t* l1_primal,
                                int32_t* blocks_dual, int32_t* blocks_primal);

/* Column-panel split of the products (option panel_split): the panels (one
 * per SM; 0 when A x̄ runs as the tiled product alone), the long rows they
 * compute in A x̄, those rows' non-zeros, the row length from which a row is
 * long, and for Aᵀy the hot rows of A whose y every panel holds and their
 * non-zeros (0 when Aᵀy runs as the tiled product alone).  No reference
 * counterpart (the reference computes A x̄ one thread per row and Aᵀy by
 * atomic scatter).  Any pointer may be NULL. */
PRAMAAN_API int pramaan_session_panel_info(pramaan_pdhg_session* s, int32_t* panels, int32_t* long_rows,
                                           int64_t* long_nnz, int32_t* min_len, int32_t* hot_rows,
                                           int64_t* hot_nnz);

#ifdef __cplusplus
}
#endif

#endif /* PRAMAAN_B200_H */
