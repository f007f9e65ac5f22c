/*
 * pdhg_oracle.c — CPU restatement of PRAMAAN's GPU PDHG path, used ONLY as
 * test infrastructure: the parity tests, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load it to check (or time beside) the CUDA
 * library.  Nothing in the product links or calls it.
 *
 * Parity pins (see tests/test_oracle_pins.py):
 *   - the reference's known answers (Wyndor 36, zero-row 5, 1-var 3,
 *     equality 5, multi -7, zero-obj 0, bounded 5; tests/test_gpu_pdhg.cpp:263-372);
 *   - the reference's own CPU check loops (cpu_spmv / cpu_spmv_t,
 *     tests/test_gpu_pdhg.cpp:147-167; cpu_pdhg_step, tests/test_pdhg_kernel.cpp:76-103);
 *   - golden trajectories recorded from the reference's GPU solver compiled
 *     for sm_100a (tests/golden/, generated by tests/golden/make_ref_golden.py).
 *
 * Arithmetic: compiled with -ffp-contract=off so every FP32 operation rounds
 * once, except where the reference's device code is contracted by nvcc into
 * an FMA; those spots call fmaf() explicitly and say so.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API __attribute__((visibility("default")))

/* LP in ModelIR form (include/pramaan/ir.hpp:62-119). */
typedef struct orc_lp {
    int32_t m, n, nnz, obj_sense; /* obj_sense: 0 min, 1 max */
    double obj_offset;
    const double* c;
    const int32_t* row_ptr;
    const int32_t* col_idx;
    const double* values;
    const double* row_lower;
    const double* row_upper;
    const double* var_lower;
    const double* var_upper;
} orc_lp;

typedef struct orc_result {
    int32_t status; /* SolveStatus values: 0 optimal, 3 iteration limit, 4 numerical failure */
    int32_t iterations;
    int32_t restarts;
    int32_t checks;
    double primal_residual;
    double dual_residual;
    double objective_value;
    double* x;            /* [n] out */
    double* row_activity; /* [m] out */
    float* y;             /* [m] out (FP32 dual iterate) */
    float* x32;           /* [n] out (FP32 primal iterate) */
} orc_result;

/* ---------------------------------------------------------------------------
 * Products
 * ------------------------------------------------------------------------ */

/* y = A x, FP32, sequential row sums: src/gpu/pdhg_kernels.cuh:24-37 and
 * tests/test_gpu_pdhg.cpp:147-156. */
ORC_API void orc_spmv_f32(int32_t m, const int32_t* rp, const int32_t* ci, const float* v,
                          const float* x, float* y) {
    for (int32_t i = 0; i < m; ++i) {
        float s = 0.0f;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
        y[i] = s;
    }
}

/* The same row sums as the GPU kernel computes them: nvcc contracts
 * `sum += values[k] * x[col_idx[k]]` (src/gpu/pdhg_kernels.cuh:32-35) into one
 * fused multiply-add per entry, in row order. */
ORC_API void orc_spmv_f32_fma(int32_t m, const int32_t* rp, const int32_t* ci, const float* v,
                              const float* x, float* y) {
    for (int32_t i = 0; i < m; ++i) {
        float s = 0.0f;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s = fmaf(v[k], x[ci[k]], s);
        y[i] = s;
    }
}

/* y = A^T x, FP32 scatter in row order: src/gpu/pdhg_kernels.cuh:42-54 (serialised)
 * and tests/test_gpu_pdhg.cpp:158-167. */
ORC_API void orc_spmv_t_f32(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                            const float* v, const float* x, float* y) {
    for (int32_t j = 0; j < n; ++j) y[j] = 0.0f;
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) y[ci[k]] += v[k] * x[i];
}

/* y = A x, FP64 (CSRMatrix::multiplyInto, include/pramaan/sparse_matrix.hpp:72-85). */
ORC_API void orc_spmv_f64(int32_t m, const int32_t* rp, const int32_t* ci, const double* v,
                          const double* x, double* y) {
    for (int32_t i = 0; i < m; ++i) {
        double s = 0.0;
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * x[ci[k]];
        y[i] = s;
    }
}

/* Counting-sort transpose (src/linalg/sparse_matrix.cpp:13-57), FP32 values. */
ORC_API void orc_transpose_f32(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                               const float* v, int32_t* trp, int32_t* tci, float* tv) {
    int32_t nnz = rp[m];
    for (int32_t j = 0; j <= n; ++j) trp[j] = 0;
    for (int32_t k = 0; k < nnz; ++k) trp[ci[k] + 1]++;
    for (int32_t j = 0; j < n; ++j) trp[j + 1] += trp[j];
    int32_t* cur = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n + 1));
    memcpy(cur, trp, sizeof(int32_t) * (size_t)(n + 1));
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            int32_t d = cur[ci[k]]++;
            tci[d] = i;
            tv[d] = v[k];
        }
    free(cur);
}

/* ---------------------------------------------------------------------------
 * Vector updates
 * ------------------------------------------------------------------------ */

/* src/gpu/pdhg_kernels.cuh:72-89 */
ORC_API void orc_dual_update(int32_t m, const float* ax, const float* sigma, const float* lr,
                             const float* ur, float* y) {
    for (int32_t i = 0; i < m; ++i) {
        const float sig = sigma[i];
        if (sig <= 0.0f) continue;
        const float w = y[i] / sig + ax[i];
        const float wp = fminf(fmaxf(w, lr[i]), ur[i]);
        y[i] = sig * (w - wp);
    }
}

/* src/gpu/pdhg_kernels.cuh:95-109.  nvcc contracts x_prev - tau*(c + ATy) and
 * 2*x_new - x_prev into FMAs; restated with fmaf. */
ORC_API void orc_primal_update(int32_t n, const float* aty, const float* tau, const float* c,
                               const float* lx, const float* ux, float* x, float* xbar) {
    for (int32_t j = 0; j < n; ++j) {
        const float x_prev = x[j];
        const float g = c[j] + aty[j];
        const float x_new = fminf(fmaxf(fmaf(-tau[j], g, x_prev), lx[j]), ux[j]);
        xbar[j] = fmaf(2.0f, x_new, -x_prev);
        x[j] = x_new;
    }
}

/* Step-1 dense iteration, src/gpu/pdhg.cu:42-66 (use_fma = 1: the device form)
 * and tests/test_pdhg_kernel.cpp:76-103 (use_fma = 0: the test's CPU form). */
ORC_API void orc_step1(int32_t n, float* x, const float* g, float tau, int32_t m, float* y,
                       const float* ax, const float* b, float sigma, int32_t use_fma) {
    for (int32_t j = 0; j < n; ++j) {
        const float u = use_fma ? fmaf(-tau, g[j], x[j]) : x[j] - tau * g[j];
        x[j] = fmaxf(0.0f, u);
    }
    for (int32_t i = 0; i < m; ++i) {
        const float d = ax[i] - b[i];
        y[i] = use_fma ? fmaf(sigma, d, y[i]) : y[i] + sigma * d;
    }
}

/* Diagonal steps, src/gpu/pdhg_solver.cu:237-250. */
ORC_API void orc_step_sizes(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                            const float* v, float* sigma, float* tau) {
    const float alpha = 0.95f;
    double* rn = (double*)calloc((size_t)(m > 0 ? m : 1), sizeof(double));
    double* cn = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = rp[i]; k < rp[i + 1]; ++k) {
            const double av = fabs((double)v[k]);
            rn[i] += av;
            cn[ci[k]] += av;
        }
    for (int32_t i = 0; i < m; ++i) sigma[i] = rn[i] > 1e-12 ? alpha / (float)rn[i] : alpha;
    for (int32_t j = 0; j < n; ++j) tau[j] = cn[j] > 1e-12 ? alpha / (float)cn[j] : alpha;
    free(rn);
    free(cn);
}

/* ComputeFp64Residuals, src/gpu/pdhg_solver.cu:107-161.  std::max(pv, viol)
 * keeps pv when viol is NaN; fmax() is used only where both operands are
 * known to be numbers, to keep that behaviour. */
static double max_keep_left(double a, double b) { return (a < b) ? b : a; }

ORC_API void orc_fp64_residuals(const orc_lp* lp, const float* v32, const float* c32,
                                const float* x, const float* y, double tol, double* out_pv,
                                double* out_dv) {
    const int32_t m = lp->m, n = lp->n;
    double* xd = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    double* act = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* aty = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int32_t j = 0; j < n; ++j) xd[j] = (double)x[j];
    orc_spmv_f64(m, lp->row_ptr, lp->col_idx, lp->values, xd, act);
    double pv = 0.0;
    for (int32_t i = 0; i < m; ++i) {
        if (act[i] < lp->row_lower[i]) pv = max_keep_left(pv, lp->row_lower[i] - act[i]);
        if (act[i] > lp->row_upper[i]) pv = max_keep_left(pv, act[i] - lp->row_upper[i]);
    }
    for (int32_t j = 0; j < n; ++j) {
        if (xd[j] < lp->var_lower[j]) pv = max_keep_left(pv, lp->var_lower[j] - xd[j]);
        if (xd[j] > lp->var_upper[j]) pv = max_keep_left(pv, xd[j] - lp->var_upper[j]);
    }
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = lp->row_ptr[i]; k < lp->row_ptr[i + 1]; ++k)
            aty[lp->col_idx[k]] += (double)v32[k] * (double)y[i];
    double cnorm = 1.0;
    for (int32_t j = 0; j < n; ++j) cnorm = max_keep_left(cnorm, (double)fabsf(c32[j]));
    double dv = 0.0;
    for (int32_t j = 0; j < n; ++j) {
        const double rc = (double)c32[j] + aty[j];
        const int at_lb = xd[j] <= lp->var_lower[j] + tol;
        const int at_ub = xd[j] >= lp->var_upper[j] - tol;
        double viol = 0.0;
        if (!at_lb && !at_ub) viol = fabs(rc);
        else if (at_lb && !at_ub) viol = max_keep_left(0.0, -rc);
        else if (at_ub && !at_lb) viol = max_keep_left(0.0, rc);
        dv = max_keep_left(dv, viol);
    }
    dv /= cnorm;
    *out_pv = pv;
    *out_dv = dv;
    free(xd);
    free(act);
    free(aty);
}

/* ---------------------------------------------------------------------------
 * The reference solve, src/gpu/pdhg_solver.cu:169-411, in FP32 on the CPU.
 * ------------------------------------------------------------------------ */
typedef struct orc_state {
    int32_t m, n;
    float *c, *lr, *ur, *lx, *ux, *sigma, *tau, *x, *y, *xbar, *ax, *aty, *v32;
} orc_state;

static void state_free(orc_state* s) {
    free(s->c); free(s->lr); free(s->ur); free(s->lx); free(s->ux); free(s->sigma);
    free(s->tau); free(s->x); free(s->y); free(s->xbar); free(s->ax); free(s->aty); free(s->v32);
}

static float* fbuf(int32_t k) { return (float*)calloc((size_t)(k > 0 ? k : 1), sizeof(float)); }

/* Conversion, steps and initial iterate (src/gpu/pdhg_solver.cu:194-297). */
static void state_init(const orc_lp* lp, orc_state* s) {
    const int32_t m = lp->m, n = lp->n, nnz = lp->nnz;
    const float kFltInf = 1e30f;
    const float obj_sign = lp->obj_sense == 1 ? -1.0f : 1.0f;
    s->m = m; s->n = n;
    s->c = fbuf(n); s->lx = fbuf(n); s->ux = fbuf(n); s->tau = fbuf(n); s->x = fbuf(n);
    s->xbar = fbuf(n); s->aty = fbuf(n);
    s->lr = fbuf(m); s->ur = fbuf(m); s->sigma = fbuf(m); s->y = fbuf(m); s->ax = fbuf(m);
    s->v32 = fbuf(nnz);
    for (int32_t j = 0; j < n; ++j) s->c[j] = (float)((double)obj_sign * lp->c[j]);
    for (int32_t i = 0; i < m; ++i) {
        s->lr[i] = (lp->row_lower[i] <= -1e29) ? -kFltInf : (float)lp->row_lower[i];
        s->ur[i] = (lp->row_upper[i] >= 1e29) ? kFltInf : (float)lp->row_upper[i];
    }
    for (int32_t j = 0; j < n; ++j) {
        s->lx[j] = (lp->var_lower[j] <= -1e29) ? -kFltInf : (float)lp->var_lower[j];
        s->ux[j] = (lp->var_upper[j] >= 1e29) ? kFltInf : (float)lp->var_upper[j];
    }
    for (int32_t k = 0; k < nnz; ++k) s->v32[k] = (float)lp->values[k];
    orc_step_sizes(m, n, lp->row_ptr, lp->col_idx, s->v32, s->sigma, s->tau);
    for (int32_t j = 0; j < n; ++j) {
        const float x0 = fmaxf(s->lx[j], fminf(0.0f, s->ux[j]));
        s->x[j] = x0;
        s->xbar[j] = x0;
    }
}

static void state_iterate(const orc_lp* lp, orc_state* s) {
    if (s->m > 0) {
        orc_spmv_f32_fma(s->m, lp->row_ptr, lp->col_idx, s->v32, s->xbar, s->ax);
        orc_dual_update(s->m, s->ax, s->sigma, s->lr, s->ur, s->y);
    }
    if (s->m > 0) orc_spmv_t_f32(s->m, s->n, lp->row_ptr, lp->col_idx, s->v32, s->y, s->aty);
    else for (int32_t j = 0; j < s->n; ++j) s->aty[j] = 0.0f;
    orc_primal_update(s->n, s->aty, s->tau, s->c, s->lx, s->ux, s->x, s->xbar);
}

/* Runs `iters` plain reference iterations from the initial iterate and
 * returns x, y, x̄ (no checks, no restarts): the trajectory used by the
 * golden-vector pins. */
ORC_API void orc_pdhg_trajectory(const orc_lp* lp, int32_t iters, float* x_out, float* y_out,
                                 float* xbar_out) {
    orc_state s;
    memset(&s, 0, sizeof(s));
    state_init(lp, &s);
    for (int32_t it = 0; it < iters; ++it) state_iterate(lp, &s);
    if (x_out) memcpy(x_out, s.x, sizeof(float) * (size_t)lp->n);
    if (y_out && lp->m > 0) memcpy(y_out, s.y, sizeof(float) * (size_t)lp->m);
    if (xbar_out) memcpy(xbar_out, s.xbar, sizeof(float) * (size_t)lp->n);
    state_free(&s);
}

ORC_API void orc_pdhg_solve_ref(const orc_lp* lp, double tol, int32_t max_iterations,
                                int32_t check_frequency, orc_result* r) {
    const int32_t m = lp->m, n = lp->n;
    r->status = 3;
    r->iterations = 0;
    r->restarts = 0;
    r->checks = 0;
    r->primal_residual = INFINITY;
    r->dual_residual = INFINITY;
    r->objective_value = 0.0;
    if (n == 0) {
        r->status = 0;
        r->objective_value = lp->obj_offset;
        if (r->row_activity) for (int32_t i = 0; i < m; ++i) r->row_activity[i] = 0.0;
        return;
    }
    for (int32_t j = 0; j < n; ++j)
        if (!isfinite(lp->c[j])) { r->status = 4; return; }
    orc_state s;
    memset(&s, 0, sizeof(s));
    state_init(lp, &s);
    double best = INFINITY;
    int stagnation = 0, restarts = 0;
    for (int32_t iter = 0; iter < max_iterations; ++iter) {
        state_iterate(lp, &s);
        if ((iter + 1) % check_frequency == 0) {
            double pv = 0, dv = 0;
            orc_fp64_residuals(lp, s.v32, s.c, s.x, s.y, tol, &pv, &dv);
            r->checks++;
            r->primal_residual = pv;
            r->dual_residual = dv;
            if (pv <= tol && dv <= tol) { r->status = 0; r->iterations = iter + 1; break; }
            const double combined = pv + dv;
            if (combined > tol * 10.0) {
                if (combined < best * 0.99) { best = combined; stagnation = 0; }
                else ++stagnation;
                if (stagnation >= 8 && restarts < 10) {
                    for (int32_t i = 0; i < m; ++i) s.y[i] = 0.0f;
                    for (int32_t j = 0; j < n; ++j) s.xbar[j] = s.x[j];
                    stagnation = 0;
                    best = INFINITY;
                    ++restarts;
                }
            }
        }
    }
    if (r->status != 0) r->iterations = max_iterations;
    r->restarts = restarts;
    {
        double pv = 0, dv = 0;
        orc_fp64_residuals(lp, s.v32, s.c, s.x, s.y, tol, &pv, &dv);
        r->primal_residual = pv;
        r->dual_residual = dv;
    }
    double obj = lp->obj_offset;
    double* xd = (double*)malloc(sizeof(double) * (size_t)n);
    for (int32_t j = 0; j < n; ++j) {
        xd[j] = (double)s.x[j];
        obj += lp->c[j] * xd[j];
    }
    r->objective_value = obj;
    if (r->x) memcpy(r->x, xd, sizeof(double) * (size_t)n);
    if (r->x32) memcpy(r->x32, s.x, sizeof(float) * (size_t)n);
    if (r->y && m > 0) memcpy(r->y, s.y, sizeof(float) * (size_t)m);
    if (r->row_activity) orc_spmv_f64(m, lp->row_ptr, lp->col_idx, lp->values, xd, r->row_activity);
    free(xd);
    state_free(&s);
}

/* ---------------------------------------------------------------------------
 * Certificate math (src/certificate/certificate.cpp:35-95): objective,
 * primal row residual, bound violation, all FP64 from the FP64 model.
 * ------------------------------------------------------------------------ */
ORC_API void orc_certificate(const orc_lp* lp, const double* x, double* obj, double* primal_res,
                             double* bound_viol) {
    const int32_t m = lp->m, n = lp->n;
    const double kInf = 1e30;
    double o = lp->obj_offset;
    for (int32_t j = 0; j < n; ++j) o += lp->c[j] * x[j];
    double* act = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    orc_spmv_f64(m, lp->row_ptr, lp->col_idx, lp->values, x, act);
    double rv = 0.0;
    for (int32_t i = 0; i < m; ++i) {
        if (lp->row_lower[i] > -kInf) { double v = lp->row_lower[i] - act[i]; if (v > rv) rv = v; }
        if (lp->row_upper[i] < kInf) { double v = act[i] - lp->row_upper[i]; if (v > rv) rv = v; }
    }
    double bv = 0.0;
    for (int32_t j = 0; j < n; ++j) {
        if (lp->var_lower[j] > -kInf) { double v = lp->var_lower[j] - x[j]; if (v > bv) bv = v; }
        if (lp->var_upper[j] < kInf) { double v = x[j] - lp->var_upper[j]; if (v > bv) bv = v; }
    }
    *obj = o;
    *primal_res = rv;
    *bound_viol = bv;
    free(act);
}

/* ---------------------------------------------------------------------------
 * Relative KKT error in FP64 (PDLP definitions, Applegate et al. 2021):
 *   primal  ||(dist(Ax, [l_r,u_r]), dist(x, [l_x,u_x]))||_2 / (1 + ||finite row bounds||_2)
 *   dual    ||rc - proj_cone(rc)||_2 / (1 + ||c||_2),  rc = c - A^T lambda
 *   gap     |p - d| / (1 + |p| + |d|)
 * with lambda = -y (the reference's y is the negated multiplier) and the
 * problem in minimisation form (c negated for maximisation).
 * out[0..2] = rel primal, rel dual, rel gap; out[3] primal obj; out[4] dual obj.
 * ------------------------------------------------------------------------ */
ORC_API void orc_rel_kkt(const orc_lp* lp, const double* x, const double* y, double* out) {
    const int32_t m = lp->m, n = lp->n;
    const double kInf = 1e29;
    const double sgn = lp->obj_sense == 1 ? -1.0 : 1.0;
    double* act = (double*)malloc(sizeof(double) * (size_t)(m > 0 ? m : 1));
    double* rc = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
    orc_spmv_f64(m, lp->row_ptr, lp->col_idx, lp->values, x, act);
    for (int32_t j = 0; j < n; ++j) rc[j] = sgn * lp->c[j];
    for (int32_t i = 0; i < m; ++i)
        for (int32_t k = lp->row_ptr[i]; k < lp->row_ptr[i + 1]; ++k)
            rc[lp->col_idx[k]] += lp->values[k] * y[i]; /* c - A^T lambda, lambda = -y */
    double rp2 = 0, b2 = 0, pobj = 0, dobj = 0, rd2 = 0, c2 = 0;
    for (int32_t i = 0; i < m; ++i) {
        const double lo = lp->row_lower[i], hi = lp->row_upper[i];
        double d = 0.0;
        if (lo > -kInf && act[i] < lo) d = lo - act[i];
        if (hi < kInf && act[i] > hi) d = act[i] - hi;
        rp2 += d * d;
        if (lo > -kInf) b2 += lo * lo;
        if (hi < kInf && !(lo > -kInf && lo == hi)) b2 += hi * hi;
        const double lam = -y[i];
        /* dual objective row terms: lambda > 0 pairs with the lower bound,
         * lambda < 0 with the upper; an infinite bound makes that sign a residual */
        if (lam > 0) { if (lo > -kInf) dobj += lam * lo; else rd2 += lam * lam; }
        else if (lam < 0) { if (hi < kInf) dobj += lam * hi; else rd2 += lam * lam; }
    }
    for (int32_t j = 0; j < n; ++j) {
        const double cj = sgn * lp->c[j];
        c2 += cj * cj;
        pobj += cj * x[j];
        const double lo = lp->var_lower[j], hi = lp->var_upper[j];
        /* x outside its bounds counts as primal residual */
        double v = 0.0;
        if (lo > -kInf && x[j] < lo) v = lo - x[j];
        if (hi < kInf && x[j] > hi) v = x[j] - hi;
        rp2 += v * v;
        const double r = rc[j];
        if (r > 0) { if (lo > -kInf) dobj += r * lo; else rd2 += r * r; }
        else if (r < 0) { if (hi < kInf) dobj += r * hi; else rd2 += r * r; }
    }
    out[0] = sqrt(rp2) / (1.0 + sqrt(b2));
    out[1] = sqrt(rd2) / (1.0 + sqrt(c2));
    out[2] = fabs(pobj - dobj) / (1.0 + fabs(pobj) + fabs(dobj));
    out[3] = pobj;
    out[4] = dobj;
    free(act);
    free(rc);
}

/* ---------------------------------------------------------------------------
 * Multi-threaded reference iteration for the CPU baseline: the same FP32
 * arithmetic as state_iterate, with A^T y as a gather over a stored
 * transpose so rows can be split across threads.
 * ------------------------------------------------------------------------ */
ORC_API int32_t orc_num_threads(void) {
#ifdef _OPENMP
    return (int32_t)omp_get_max_threads();
#else
    return 1;
#endif
}

ORC_API void orc_set_num_threads(int32_t t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

ORC_API void orc_pdhg_iterations_mt(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                                    const float* v, const int32_t* trp, const int32_t* tci,
                                    const float* tv, const float* sigma, const float* lr,
                                    const float* ur, const float* tau, const float* c,
                                    const float* lx, const float* ux, float* x, float* xbar,
                                    float* y, int32_t iters) {
    for (int32_t it = 0; it < iters; ++it) {
#pragma omp parallel for schedule(dynamic, 1024)
        for (int32_t i = 0; i < m; ++i) {
            float s = 0.0f;
            for (int32_t k = rp[i]; k < rp[i + 1]; ++k) s += v[k] * xbar[ci[k]];
            const float sig = sigma[i];
            if (sig <= 0.0f) continue;
            const float w = y[i] / sig + s;
            const float wp = fminf(fmaxf(w, lr[i]), ur[i]);
            y[i] = sig * (w - wp);
        }
#pragma omp parallel for schedule(dynamic, 1024)
        for (int32_t j = 0; j < n; ++j) {
            float s = 0.0f;
            for (int32_t k = trp[j]; k < trp[j + 1]; ++k) s += tv[k] * y[tci[k]];
            const float x_prev = x[j];
            const float x_new = fminf(fmaxf(fmaf(-tau[j], c[j] + s, x_prev), lx[j]), ux[j]);
            xbar[j] = fmaf(2.0f, x_new, -x_prev);
            x[j] = x_new;
        }
    }
}
