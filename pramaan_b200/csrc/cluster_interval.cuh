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
// records were packed from): one thread per row (kRowsPerPass rows of a thread
// advanced together, kEntryChunk entries at a time), entries in CSR order, one
// FMA each, so a row's sum has the order the tiled kernel uses for a row inside
// one tile.  The vector updates are the same epilogue objects as the tiled
// path (same arithmetic per element).  The gathers of y and x̄, written by the
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

// Rows r_u = r0 + u * step (u < kRowsPerPass, those below r_end) of a flat
// CSR times x, into acc[u]: each row's entries in CSR order, one FMA each.
// The entries are loaded kEntryChunk at a time for every row of the pass
// before any of them is summed, so one chunk costs one round trip of
// dependent loads (column index, then x) whatever the row lengths, and long
// rows (a capacity row touches every product of its period) take
// ceil(length / kEntryChunk) round trips instead of one per entry.  x is
// read past L1 (other SMs of the cluster wrote it); the operand is read-only
// for the kernel.
constexpr int kRowsPerPass = 2;
constexpr int kEntryChunk = 8;

__device__ __forceinline__ void flat_rows_dot(const FlatCsr& A, const float* __restrict__ x, int r0, int step,
                                              int r_end, float (&acc)[kRowsPerPass]) {
    int e[kRowsPerPass], e1[kRowsPerPass];
    bool more = false;
#pragma unroll
    for (int u = 0; u < kRowsPerPass; ++u) {
        const int r = r0 + u * step;
        const bool ok = r < r_end;
        e[u] = ok ? __ldg(A.row_ptr + r) : 0;
        e1[u] = ok ? __ldg(A.row_ptr + r + 1) : 0;
        acc[u] = 0.0f;
        more = more || e[u] < e1[u];
    }
    while (more) {
        float v[kRowsPerPass][kEntryChunk], xv[kRowsPerPass][kEntryChunk];
        int c[kRowsPerPass][kEntryChunk];
#pragma unroll
        for (int u = 0; u < kRowsPerPass; ++u)
#pragma unroll
            for (int k = 0; k < kEntryChunk; ++k) {
                const bool ok = e[u] + k < e1[u];
                c[u][k] = ok ? __ldg(A.col + e[u] + k) : 0;
                v[u][k] = ok ? __ldg(A.val + e[u] + k) : 0.0f;
            }
#pragma unroll
        for (int u = 0; u < kRowsPerPass; ++u)
#pragma unroll
            for (int k = 0; k < kEntryChunk; ++k)
                xv[u][k] = e[u] + k < e1[u] ? __ldcg(x + c[u][k]) : 0.0f;
        more = false;
#pragma unroll
        for (int u = 0; u < kRowsPerPass; ++u) {
#pragma unroll
            for (int k = 0; k < kEntryChunk; ++k)
                if (e[u] + k < e1[u]) acc[u] = fmaf(v[u][k], xv[u][k], acc[u]);
            e[u] += kEntryChunk;
            more = more || e[u] < e1[u];
        }
    }
}

// Grid: (number of LPs) x C blocks of kClusterThreads, clusters of C blocks
// along x; cluster q runs the LP with rows [lps[q].x, lps[q].y) and columns
// [lps[q].z, lps[q].w) of the current layout.  fpr_*: the fixed-point residual terms of
// the interval's first (…0) and last (…1) iteration, as the tiled path writes
// them.
__global__ void __launch_bounds__(kClusterThreads)
    halpern_cluster_kernel(const int4* __restrict__ lps, FlatCsr A, FlatCsr AT, EpiPrimalHalpern ep,
                           EpiDualHalpern ed, const float* y, const float* xbar, int iters, double* fpr_c0,
                           double* fpr_c1, double* fpr_r0, double* fpr_r1) {
    const int4 L = lps[cluster_index_x()];
    const int nth = int(cluster_blocks()) * blockDim.x;
    const int tid = int(cluster_rank_in()) * blockDim.x + threadIdx.x;
    typename EpiPrimalHalpern::State sp;
    typename EpiDualHalpern::State sd;
    ep.init(sp);
    ed.init(sd);
    for (int it = 0; it < iters; ++it) {
        ep.offset = it;
        ep.fpr = it == 0 ? fpr_c0 : (it == iters - 1 ? fpr_c1 : nullptr);
        ed.offset = it;
        ed.fpr = it == 0 ? fpr_r0 : (it == iters - 1 ? fpr_r1 : nullptr);
        for (int j0 = L.z + tid; j0 < L.w; j0 += nth * kRowsPerPass) {
            float acc[kRowsPerPass];
            flat_rows_dot(AT, y, j0, nth, L.w, acc);
#pragma unroll
            for (int u = 0; u < kRowsPerPass; ++u)
                if (j0 + u * nth < L.w) ep.apply(sp, j0 + u * nth, acc[u]);
        }
        cluster_barrier();
        for (int i0 = L.x + tid; i0 < L.y; i0 += nth * kRowsPerPass) {
            float acc[kRowsPerPass];
            flat_rows_dot(A, xbar, i0, nth, L.y, acc);
#pragma unroll
            for (int u = 0; u < kRowsPerPass; ++u)
                if (i0 + u * nth < L.y) ed.apply(sd, i0 + u * nth, acc[u]);
        }
        cluster_barrier();
    }
    ep.finish(sp, 0);
    ed.finish(sd, 0);
}

}  // namespace pb
