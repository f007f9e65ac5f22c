// interval.cuh — a whole check interval of the Halpern iteration in one
// cooperative launch (small operands).
//
// For operands of a few thousand tiles each product is a latency chain of a
// few microseconds (bulk copy, gathers, epilogue) and launching two kernels
// per iteration costs as much again.  This kernel keeps one grid resident for
// all iterations of a check interval: per iteration the primal product over
// A^T (EpiPrimalHalpern), the fixup of its crossing / empty rows, the dual
// product over A (EpiDualHalpern) and its fixup, separated by grid barriers.
// The first bulk copies of every product are issued before the barrier that
// precedes it (tile records are never written), so they overlap the wait.
// Every warp processes the same tiles in every product (same grid), so the
// results are bit-identical to the per-kernel path.
#pragma once

#include "adaptive.cuh"
#include "spmv.cuh"

namespace pb {

struct GridSync {
    unsigned* count;    // arrivals at the current barrier
    unsigned* gen;      // barrier generation
    unsigned nblocks;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier for a cooperative launch.  Every block calls it the same
// number of times.  Arrival is an acquire-release add on the counter (the
// block's writes, ordered before it by __syncthreads, are released with it);
// the last block resets the counter and releases the next generation, the
// others poll it with acquire loads.  The wait is bounded (kWaitLimitNs): a
// block that gives up, or enters with ok_in false, sets the status word's
// error bit and returns false, and the other blocks then give up at their next
// barrier at the latest, so the grid leaves the interval within a time limit.
__device__ __forceinline__ bool grid_sync(const GridSync& g, bool ok_in, int* status) {
    __shared__ int s_ok;
    const bool block_ok = __syncthreads_and(ok_in);
    if (threadIdx.x == 0) {
        int ok = block_ok ? 1 : 0;
        if (!block_ok) atomicOr(status, kDevErrTimeout);
        const unsigned gen0 = ld_acquire_u32(g.gen);
        unsigned prev;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(prev) : "l"(g.count) : "memory");
        if (prev == g.nblocks - 1) {
            asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(g.count) : "memory");
            asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(g.gen) : "memory");
        } else {
            unsigned spins = 0;
            unsigned long long t0 = 0;
            while (ld_acquire_u32(g.gen) == gen0) {
                if ((++spins & 63u) == 0u) {
                    const unsigned long long t = global_timer_ns();
                    if (t0 == 0) t0 = t;
                    else if (t - t0 > kWaitLimitNs) {
                        ok = 0;
                        atomicOr(status, kDevErrTimeout);
                        break;
                    }
                }
            }
            if (ok && (ld_acquire_u32(reinterpret_cast<const unsigned*>(status)) & unsigned(kDevErrTimeout))) ok = 0;
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

template <bool kMapA, bool kMapAT>
__global__ void __launch_bounds__(kSpmvWarps * 32)
    halpern_interval_kernel(const CsrView A, const CsrView AT, EpiPrimalHalpern ep, EpiDualHalpern ed,
                            const float* __restrict__ y, const float* __restrict__ xbar, int iters,
                            double* fpr_c0, double* fpr_c1, double* fpr_r0, double* fpr_r1, GridSync gs,
                            int* status) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint32_t used = 0;
    bool ok = true;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x;
    const int nth = gridDim.x * blockDim.x;
    const bool fixA = A.num_cross + A.num_empty > 0;
    const bool fixAT = AT.num_cross + AT.num_empty > 0;
    for (int it = 0; it < iters && ok; ++it) {
        ep.offset = it;
        ep.fpr = it == 0 ? fpr_c0 : (it == iters - 1 ? fpr_c1 : nullptr);
        ed.offset = it;
        ed.fpr = it == 0 ? fpr_r0 : (it == iters - 1 ? fpr_r1 : nullptr);
        // primal: x+ from A^T y (y of the previous iteration's dual product)
        ok = spmv_tiles<EpiPrimalHalpern, float, float, false, kMapAT, kSpmvWarps, kSpmvStages>(
            AT, y, ep, status, smem, used, it == 0, [&] { return it == 0 ? true : grid_sync(gs, true, status); });
        ok = __syncthreads_and(ok);
        if (fixAT) {
            ok = grid_sync(gs, ok, status);
            if (!ok) break;
            spmv_fixup_rows<EpiPrimalHalpern, float>(AT, ep, tid, nth);
        }
        // dual: y from A x_bar (x_bar complete only after the barrier)
        const bool ok_in = ok;
        ok = spmv_tiles<EpiDualHalpern, float, float, false, kMapA, kSpmvWarps, kSpmvStages>(
            A, xbar, ed, status, smem, used, false, [&] { return grid_sync(gs, ok_in, status); });
        ok = __syncthreads_and(ok);
        if (fixA) {
            ok = grid_sync(gs, ok, status);
            if (!ok) break;
            spmv_fixup_rows<EpiDualHalpern, float>(A, ed, tid, nth);
        }
    }
}

}  // namespace pb
