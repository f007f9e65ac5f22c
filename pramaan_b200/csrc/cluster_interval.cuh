// cluster_interval.cuh — a whole check interval of the batched Halpern
// iteration in one launch, one thread-block cluster per LP.
//
// The LPs of a batch are independent: nothing but the launch boundary forces
// LP a to wait for LP b.  Here every LP of the current layout gets its own
// cluster of C blocks (one or more SMs), which runs all iterations of the
// check interval on its own: the primal half (A^T y and EpiPrimalHalpern for
// the LP's columns), a cluster barrier, the dual half (A x̄ and EpiDualHalpern
// for its rows), a cluster barrier.  There is no grid-wide barrier and no
// launch per iteration, so an LP that is left alone in the batch (the slow
// tail) iterates at the latency of two small products on C SMs instead of
// four dependent kernel launches across the GPU, and a small LP's operand and
// vectors stay in L2 for the whole interval instead of being streamed again
// every iteration.
//
// The products read the flat FP32 CSR of A and of A^T (the operand the tile
// records were packed from): one thread per short row (a few rows of a thread
// advanced together, a chunk of entries at a time), entries in CSR order, one
// FMA each, so a short row's sum has the order the tiled kernel uses for a row
// inside one tile; one warp per long row.  The vector updates are the same
// epilogue objects as the tiled path (same arithmetic per element).  The
// gathers of y and x̄, written by the
// other blocks of the cluster, are ld.global.cg loads after the cluster
// barrier (barrier.cluster.arrive.release / wait.acquire order the writes
// before it and the reads after it); every other vector an element reads is
// either constant for the interval or the element's own, written by the same
// thread.  Every thread of a cluster runs the same number of barriers.
#pragma once

#include "adaptive.cuh"

namespace pb {

constexpr int kClusterThreads = 512;    // threads per block of the cluster kernel
constexpr int kClusterMax = 16;         // largest cluster (non-portable size)

struct FlatCsr {
    const int* row_ptr;
    const int* col;
    const float* val;
};

__device__ __forceinline__ unsigned cluster_rank_in() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_blocks() {
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ unsigned cluster_index_x() {
    unsigned r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_barrier() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// Rows r_u = r0 + u * step (u < kRows, those below r_end) of a flat CSR
// times x, into acc[u]: each row's entries in CSR order, one FMA each.  The
// entries are loaded kChunk at a time for every row of the pass before any of
// them is summed, so one chunk costs one round trip of dependent loads
// (column index, then x) whatever the row lengths.  Rows longer than
// kClusterLongRow are left to the warps of cluster_half (own[u] false): a thread
// would need one round trip per kChunk of their entries, and the slowest
// thread sets the time of the half-iteration for the whole cluster.  x is
// read past L1 (other SMs of the cluster wrote it); the operand is read-only
// for the kernel.
constexpr int kClusterLongRow = 16;

template <int kRows, int kChunk>
__device__ __forceinline__ void flat_rows_dot(const FlatCsr& A, const float* __restrict__ x, int r0, int step,
                                              int r_end, float (&acc)[kRows], bool (&own)[kRows]) {
    int e[kRows], e1[kRows];
    bool more = false;
#pragma unroll
    for (int u = 0; u < kRows; ++u) {
        const int r = r0 + u * step;
        const bool ok = r < r_end;
        e[u] = ok ? __ldg(A.row_ptr + r) : 0;
        e1[u] = ok ? __ldg(A.row_ptr + r + 1) : 0;
        own[u] = ok && e1[u] - e[u] <= kClusterLongRow;
        if (!own[u]) e1[u] = e[u];
        acc[u] = 0.0f;
        more = more || e[u] < e1[u];
    }
    while (more) {
        float v[kRows][kChunk], xv[kRows][kChunk];
        int c[kRows][kChunk];
#pragma unroll
        for (int u = 0; u < kRows; ++u)
#pragma unroll
            for (int k = 0; k < kChunk; ++k) {
                const bool ok = e[u] + k < e1[u];
                c[u][k] = ok ? __ldg(A.col + e[u] + k) : 0;
                v[u][k] = ok ? __ldg(A.val + e[u] + k) : 0.0f;
            }
#pragma unroll
        for (int u = 0; u < kRows; ++u)
#pragma unroll
            for (int k = 0; k < kChunk; ++k)
                xv[u][k] = e[u] + k < e1[u] ? __ldcg(x + c[u][k]) : 0.0f;
        more = false;
#pragma unroll
        for (int u = 0; u < kRows; ++u) {
#pragma unroll
            for (int k = 0; k < kChunk; ++k)
                if (e[u] + k < e1[u]) acc[u] = fmaf(v[u][k], xv[u][k], acc[u]);
            e[u] += kChunk;
            more = more || e[u] < e1[u];
        }
    }
}

// One half-iteration of one LP on its cluster: rows [r_begin, r_end) of A
// times x, each row's update by ep.  Short rows: a thread per row, kRows rows
// of a thread advanced together; every row's epilogue inputs are loaded
// before its products (they do not depend on it), so their round trips
// overlap the product's.  Long rows (long_rows[l_begin..l_end), the rows of
// the range longer than kClusterLongRow, listed by the host): a warp per row,
// lane k summing entries k, k + 32, … in CSR order, then a fixed xor-tree of
// shuffles, lane 0 applying the update.  Every row is updated exactly once.
template <int kRows, int kChunk, class Epi>
__device__ __forceinline__ void cluster_half(const FlatCsr& A, const float* __restrict__ x, int r_begin, int r_end,
                                             const int* __restrict__ long_rows, int l_begin, int l_end, int tid,
                                             int nth, const Epi& ep, typename Epi::State& st, float w) {
    for (int r0 = r_begin + tid; r0 < r_end; r0 += nth * kRows) {
        typename Epi::In in[kRows];
#pragma unroll
        for (int u = 0; u < kRows; ++u)
            if (r0 + u * nth < r_end) in[u] = ep.load(r0 + u * nth, w);
        float acc[kRows];
        bool own[kRows];
        flat_rows_dot<kRows, kChunk>(A, x, r0, nth, r_end, acc, own);
#pragma unroll
        for (int u = 0; u < kRows; ++u)
            if (own[u]) ep.store(st, r0 + u * nth, in[u], acc[u]);
    }
    const int lane = tid & 31;
    for (int i = l_begin + (tid >> 5); i < l_end; i += nth >> 5) {
        const int r = __ldg(long_rows + i);
        const typename Epi::In in = ep.load(r, w);
        const int e1 = __ldg(A.row_ptr + r + 1);
        float acc = 0.0f;
        for (int e = __ldg(A.row_ptr + r) + lane; e < e1; e += 64) {
            const bool two = e + 32 < e1;
            const int c0 = __ldg(A.col + e);
            const float v0 = __ldg(A.val + e);
            const int c1 = two ? __ldg(A.col + e + 32) : 0;
            const float v1 = two ? __ldg(A.val + e + 32) : 0.0f;
            const float x0 = __ldcg(x + c0);
            const float x1 = two ? __ldcg(x + c1) : 0.0f;
            acc = fmaf(v0, x0, acc);
            if (two) acc = fmaf(v1, x1, acc);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) ep.store(st, r, in, acc);
    }
}

// Grid: (number of LPs) x C blocks of kClusterThreads, clusters of C blocks
// along x; cluster q runs the LP with rows [lps[q].x, lps[q].y) and columns
// [lps[q].z, lps[q].w) of the current layout.  Its long rows of A are
// long_a[lr[q].x .. lr[q].y) and its long rows of A^T (columns)
// long_at[lr[q].z .. lr[q].w).  fpr_*: the fixed-point residual terms of the
// interval's first (…0) and last (…1) iteration, as the tiled path writes
// them.  A column of a rolling-horizon LP has two or three entries and a row
// about six, hence four rows of four-entry chunks per thread in the primal
// half and two rows of eight in the dual half.
__global__ void __launch_bounds__(kClusterThreads)
    halpern_cluster_kernel(const int4* __restrict__ lps, const int4* __restrict__ lr, const int* __restrict__ long_a,
                           const int* __restrict__ long_at, FlatCsr A, FlatCsr AT, EpiPrimalHalpern ep,
                           EpiDualHalpern ed, const float* y, const float* xbar, int iters, double* fpr_c0,
                           double* fpr_c1, double* fpr_r0, double* fpr_r1) {
    const int4 L = lps[cluster_index_x()];
    const int4 R = lr[cluster_index_x()];
    const int nth = int(cluster_blocks()) * blockDim.x;
    const int tid = int(cluster_rank_in()) * blockDim.x + threadIdx.x;
    typename EpiPrimalHalpern::State sp;
    typename EpiDualHalpern::State sd;
    ep.init(sp);
    ed.init(sd);
    // the cluster's LP (every row and column of the cluster belongs to it), so
    // the Halpern weight is one value per iteration
    const int q = ep.lp && L.z < L.w ? __ldg(ep.lp + L.z) : (ed.lp && L.x < L.y ? __ldg(ed.lp + L.x) : 0);
    for (int it = 0; it < iters; ++it) {
        ep.offset = it;
        ep.fpr = it == 0 ? fpr_c0 : (it == iters - 1 ? fpr_c1 : nullptr);
        ed.offset = it;
        ed.fpr = it == 0 ? fpr_r0 : (it == iters - 1 ? fpr_r1 : nullptr);
        const float w = halpern_weight_lp(ep.iter_base, it, ep.restart_iter, q);
        cluster_half<4, 4>(AT, y, L.z, L.w, long_at, R.z, R.w, tid, nth, ep, sp, w);
        cluster_barrier();
        cluster_half<2, 8>(A, xbar, L.x, L.y, long_a, R.x, R.y, tid, nth, ed, sd, w);
        cluster_barrier();
    }
    ep.finish(sp, 0);
    ed.finish(sd, 0);
}

}  // namespace pb
