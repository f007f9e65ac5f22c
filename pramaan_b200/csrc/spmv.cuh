// spmv.cuh — nnz-balanced ("merge-path") CSR SpMV for sm_100a with a fused
// per-row epilogue.
//
// Replaces the reference's csr_spmv_kernel (src/gpu/pdhg_kernels.cuh:24-37,
// one thread per row) and csr_spmv_t_kernel (:42-54, atomic scatter).  The
// transpose product is run by the same kernel over a stored transpose, so
// both products are gathers and both are deterministic run to run.
//
// Tiled operand format (built once per matrix, see csr_device.cu)
//   The non-zeros are cut into tiles of T = BLOCK*IPT consecutive entries.
//   Per tile, four slabs sit at 16-byte aligned offsets:
//     col   int32[T]      column indices
//     val   fp32 [T]      values (FP32-rounded)      [+ val_lo fp32[T]]
//     flags u32 [T/32]    bit q set <=> entry q starts a row
//     meta  int4          {first_row, head_t0, tail_span, tail_continues}
//   Empty rows are compacted out (an optional row_map gives the original row
//   of every compacted row; empty rows get their epilogue from a separate
//   pass), and the padding after the last entry forms a virtual row that is
//   never emitted.  Row ids therefore follow from the bitmap alone:
//   row(q) = first_row + #starts in (0, q], and the kernel never reads
//   row_ptr.
//
// Schedule
//   A persistent grid (a multiple of the SM count) walks the tiles with a
//   static stride.  Thread 0 streams every tile's four slabs into a
//   STAGES-deep shared-memory ring with 1-D TMA bulk copies
//   (cp.async.bulk ... mbarrier::complete_tx, L2 evict_first) while the
//   block works on earlier tiles; waits on the ring's mbarriers are bounded.
//   Every thread owns IPT consecutive entries.  Row ids come from popcounts
//   of the bitmap (warp shuffles, no block barrier), the epilogue's vectors
//   for the rows a thread will finish are prefetched into L2 together with
//   the x gathers, and one segmented block scan (shuffles + one barrier)
//   carries open-row partial sums across threads.  A row that crosses tile
//   boundaries is finished by the "last arriver": each tile holding a piece
//   stores its partial in carry[], bumps the row's counter with an acq_rel
//   atomic, and the tile that completes the count adds the pieces in tile
//   order.  No block ever waits on another block, and every sum has a fixed
//   order, so results are bit-identical between runs.
#pragma once

#include "common.cuh"

namespace pb {

// Device view of one CSR operand in the tiled format.
struct CsrView {
    int rows = 0;          // original rows (epilogue index space)
    int cols = 0;
    int nnz = 0, nnz_pad = 0, num_tiles = 0;
    int rows_c = 0;        // non-empty (compacted) rows
    int num_empty = 0;     // rows without entries
    const int* col = nullptr;        // nnz_pad
    const float* val = nullptr;      // nnz_pad
    const float* val_lo = nullptr;   // nnz_pad or null
    const uint32_t* flags = nullptr; // nnz_pad / 32
    const int4* meta = nullptr;      // num_tiles
    const int* row_map = nullptr;    // rows_c (null: identity)
    const int* empty_rows = nullptr; // num_empty
    void* carry = nullptr;           // 2 * num_tiles accumulators (8-byte slots)
    int* counter = nullptr;          // num_tiles, zero between launches
};

constexpr int kSpmvBlock = 256;
constexpr int kSpmvIpt = 8;
constexpr int kSpmvTile = kSpmvBlock * kSpmvIpt;
constexpr int kSpmvStages = 4;

template <int BLOCK, int IPT, int STAGES, bool kLo, typename AccT>
struct SpmvSmemLayout {
    static constexpr int T = BLOCK * IPT;
    static constexpr int NW = BLOCK / 32;
    static constexpr int kArrays = kLo ? 3 : 2;
    static constexpr size_t flag_bytes = size_t(T) / 8;
    static constexpr size_t stage_bytes = size_t(T) * 4 * kArrays + flag_bytes + 16;
    static constexpr size_t off_col = 0;
    static constexpr size_t off_val = off_col + size_t(STAGES) * T * 4;
    static constexpr size_t off_lo = off_val + size_t(STAGES) * T * 4;
    static constexpr size_t off_flags = off_val + size_t(STAGES) * T * 4 * (kArrays - 1);
    static constexpr size_t off_meta = off_flags + size_t(STAGES) * flag_bytes;
    static constexpr size_t off_bar = off_meta + size_t(STAGES) * 16;
    static constexpr size_t off_wf = off_bar + size_t(STAGES) * 8;
    static constexpr size_t off_wv = off_wf + 8 * ((size_t(NW) * 4 + 7) / 8);
    static constexpr size_t bytes = ((off_wv + size_t(NW) * sizeof(AccT)) + 127) / 128 * 128;
    static constexpr unsigned tx_bytes = unsigned(stage_bytes);
    static_assert(T % 32 == 0 && 32 % IPT == 0, "IPT must divide 32");
    static_assert((size_t(T) * 4) % 16 == 0 && flag_bytes % 16 == 0, "TMA slabs must be 16-byte multiples");
};

// Epilogue concept:
//   struct Epi {
//     struct State {...};                                  // per-thread state
//     __device__ void init(State&) const;
//     __device__ void prefetch(int row) const;             // L2 prefetch of row data
//     __device__ void apply(State&, int row, AccT value) const;   // row complete
//     __device__ void finish(State&) const;                // once by every thread at exit
//   };

__device__ __forceinline__ int atomic_add_acq_rel_gpu(int* p, int v) {
    int old;
    asm volatile("atom.acq_rel.gpu.global.add.s32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

template <typename T>
__device__ __forceinline__ T ld_relaxed_gpu(const T* p);
template <>
__device__ __forceinline__ float ld_relaxed_gpu<float>(const float* p) {
    float v;
    asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
    return v;
}
template <>
__device__ __forceinline__ double ld_relaxed_gpu<double>(const double* p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

template <typename AccT>
struct SegPair {   // (row end seen, open-row partial)
    int f;
    AccT v;
};

template <class Epi, typename AccT, typename XT, bool kLo, bool kRowMap, int BLOCK, int IPT, int STAGES>
__global__ void __launch_bounds__(BLOCK)
    spmv_tile_kernel(const CsrView A, const XT* __restrict__ x, const Epi epi,
                     int* __restrict__ dev_status) {
    using L = SpmvSmemLayout<BLOCK, IPT, STAGES, kLo, AccT>;
    constexpr int T = L::T;
    constexpr int NW = L::NW;
    constexpr int WPT = T / 32;              // flag words per tile
    constexpr unsigned kMask = (IPT == 32) ? 0xffffffffu : ((1u << IPT) - 1u);

    extern __shared__ __align__(128) unsigned char smem[];
    int* s_col = reinterpret_cast<int*>(smem + L::off_col);
    float* s_val = reinterpret_cast<float*>(smem + L::off_val);
    float* s_lo = reinterpret_cast<float*>(smem + L::off_lo);
    uint32_t* s_flags = reinterpret_cast<uint32_t*>(smem + L::off_flags);
    int4* s_meta = reinterpret_cast<int4*>(smem + L::off_meta);
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem + L::off_bar);
    int* s_wf = reinterpret_cast<int*>(smem + L::off_wf);
    AccT* s_wv = reinterpret_cast<AccT*>(smem + L::off_wv);

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int rows_c = A.rows_c;
    const unsigned last_col = static_cast<unsigned>(A.cols - 1);

    typename Epi::State est;
    epi.init(est);

    const int nt = A.num_tiles;
    const int first = blockIdx.x;
    const int stride = gridDim.x;
    const int mine = first < nt ? (nt - first + stride - 1) / stride : 0;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) mbar_init(&s_bar[s], 1);
        fence_mbar_init();
    }
    __syncthreads();

    uint64_t policy = 0;
    if (tid == 0) policy = l2_policy_evict_first();

    auto issue = [&](int i) {
        const int t = first + i * stride;
        const int s = i % STAGES;
        const size_t off = size_t(t) * T;
        mbar_arrive_expect_tx(&s_bar[s], L::tx_bytes);
        tma_bulk_g2s(s_col + s * T, A.col + off, T * 4, &s_bar[s], policy);
        tma_bulk_g2s(s_val + s * T, A.val + off, T * 4, &s_bar[s], policy);
        if constexpr (kLo) tma_bulk_g2s(s_lo + s * T, A.val_lo + off, T * 4, &s_bar[s], policy);
        tma_bulk_g2s(s_flags + s * WPT, A.flags + size_t(t) * WPT, unsigned(L::flag_bytes), &s_bar[s], policy);
        tma_bulk_g2s(s_meta + s, A.meta + t, 16, &s_bar[s], policy);
    };

    if (tid == 0) {
        fence_proxy_async_smem();
        const int pre = mine < STAGES - 1 ? mine : STAGES - 1;
        for (int i = 0; i < pre; ++i) issue(i);
    }

    AccT* carry = reinterpret_cast<AccT*>(A.carry);
    bool failed = false;
    int i = 0;
    for (; i < mine; ++i) {
        const int t = first + i * stride;
        const int s = i % STAGES;
        const uint32_t parity = (i / STAGES) & 1;
        if (tid == 0 && i + STAGES - 1 < mine) {
            fence_proxy_async_smem();
            issue(i + STAGES - 1);
        }
        const bool ok = mbar_wait_bounded(&s_bar[s], parity);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }

        const int4 meta = s_meta[s];   // first_row, head_t0, tail_span, tail_continues
        const uint32_t* fl = s_flags + s * WPT;
        const int q0 = tid * IPT;      // tile-local index of my first entry

        // ---- row-start bits of my entries and of the entry after them ----
        const uint32_t my = (fl[q0 >> 5] >> (q0 & 31)) & kMask;
        uint32_t next_start;
        if (tid == BLOCK - 1) next_start = meta.w ? 0u : 1u;
        else next_start = (fl[(q0 + IPT) >> 5] >> ((q0 + IPT) & 31)) & 1u;
        const uint32_t ends = (my >> 1) | (next_start << (IPT - 1));   // bit j: entry j ends a row

        // ---- row id of my first entry: first_row + #starts in (0, q0] ----
        int row0;
        {
            // starts in tile entries [0, q0): popcount of the warps before me + lanes before me
            int before_warp = 0;
            const int words_before = warp * (32 * IPT / 32);
            for (int w = lane; w < words_before; w += 32) before_warp += __popc(fl[w]);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) before_warp += __shfl_xor_sync(0xffffffffu, before_warp, o);
            int incl = __popc(my);
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const int v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= d) incl += v;
            }
            const int starts_lt_q0 = before_warp + incl - __popc(my);
            const int s0 = fl[0] & 1u;
            // #starts in (0, q0] = starts in [0, q0] minus the start at entry 0
            row0 = meta.x + (starts_lt_q0 + (my & 1u)) - s0;
        }
        const bool head_before = (my & 1u) == 0;   // my first row began before my first entry

        // ---- prefetch the epilogue rows I will finish, then gather x ----
        const int nends = __popc(ends);
        if (nends > 0 && !kRowMap) {
            const int r_first = row0;
            const int r_last = row0 + nends - 1;
            if (r_first < rows_c) epi.prefetch(r_first);
            if (r_last != r_first && r_last < rows_c) epi.prefetch(r_last);
        }
        AccT p[IPT];
        {
            const int* sc = s_col + s * T + q0;
            const float* sv = s_val + s * T + q0;
#pragma unroll
            for (int j = 0; j < IPT; j += 4) {
                const int4 c4 = *reinterpret_cast<const int4*>(sc + j);
                const float4 v4 = *reinterpret_cast<const float4*>(sv + j);
                const int cc[4] = {c4.x, c4.y, c4.z, c4.w};
                const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
                float ll[4] = {0.f, 0.f, 0.f, 0.f};
                if constexpr (kLo) {
                    const float4 l4 = *reinterpret_cast<const float4*>(s_lo + s * T + q0 + j);
                    ll[0] = l4.x; ll[1] = l4.y; ll[2] = l4.z; ll[3] = l4.w;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    unsigned ci = static_cast<unsigned>(cc[q]);
                    ci = ci < last_col ? ci : last_col;   // never gather out of bounds
                    const XT xv = __ldg(x + ci);
                    if constexpr (kLo) {
                        p[j + q] = (static_cast<AccT>(vv[q]) + static_cast<AccT>(ll[q])) *
                                   static_cast<AccT>(xv);
                    } else {
                        p[j + q] = static_cast<AccT>(vv[q]) * static_cast<AccT>(xv);
                    }
                }
            }
        }

        auto emit = [&](int row_c, AccT v) {
            if (row_c >= rows_c) return;   // virtual padding row
            const int r = kRowMap ? A.row_map[row_c] : row_c;
            epi.apply(est, r, v);
        };

        // ---- walk my entries; finish the rows that end here ----
        AccT acc = AccT(0);
        int cur = row0;
        int nemit = 0;
        AccT head_acc = AccT(0);
        bool head_pending = false;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            acc += p[j];
            if ((ends >> j) & 1u) {
                if (nemit == 0 && head_before) { head_acc = acc; head_pending = true; }
                else emit(cur, acc);
                ++nemit;
                ++cur;
                acc = AccT(0);
            }
        }

        // ---- segmented block scan of (row end seen, open partial) ----
        SegPair<AccT> a{nemit > 0 ? 1 : 0, acc};
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int fo = __shfl_up_sync(0xffffffffu, a.f, d);
            const AccT vo = __shfl_up_sync(0xffffffffu, a.v, d);
            if (lane >= d) { if (!a.f) a.v += vo; a.f |= fo; }
        }
        if (lane == 31) { s_wf[warp] = a.f; s_wv[warp] = a.v; }
        __syncthreads();
        SegPair<AccT> pre{0, AccT(0)};
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            if (w < warp) {
                const int fw = s_wf[w];
                const AccT vw = s_wv[w];
                if (fw) { pre.f = 1; pre.v = vw; } else { pre.v += vw; }
            }
        }
        SegPair<AccT> ex;   // exclusive: partial of the row open at my first entry
        {
            const int fo = __shfl_up_sync(0xffffffffu, a.f, 1);
            const AccT vo = __shfl_up_sync(0xffffffffu, a.v, 1);
            if (lane == 0) ex = pre;
            else { ex.f = pre.f | fo; ex.v = fo ? vo : pre.v + vo; }
        }
        const AccT carry_in = ex.v;

        auto arrive = [&](int row_c, AccT v, bool is_tail, int slot, int count) {
            carry[2 * t + (is_tail ? 1 : 0)] = v;
            const int old = atomic_add_acq_rel_gpu(&A.counter[slot], 1);
            if (old == count - 1) {
                AccT sum = ld_relaxed_gpu(&carry[2 * slot + 1]);
                for (int tt = slot + 1; tt < slot + count; ++tt) sum += ld_relaxed_gpu(&carry[2 * tt]);
                A.counter[slot] = 0;
                emit(row_c, sum);
            }
        };

        // first row finished by this thread began before my first entry
        if (head_pending) {
            const AccT tot = head_acc + carry_in;
            if (row0 == meta.x && meta.y >= 0) {
                // it began in an earlier tile: this tile holds its last piece
                const int slot = meta.y;
                arrive(row0, tot, false, slot, A.meta[slot].z);
            } else {
                emit(row0, tot);
            }
        }
        // the tile's last row continues into the next tile
        if (tid == BLOCK - 1 && meta.w) {
            const AccT tot = nemit > 0 ? acc : carry_in + acc;
            if (cur == meta.x && meta.y >= 0) {
                const int slot = meta.y;   // a middle piece of a row begun earlier
                arrive(cur, tot, false, slot, A.meta[slot].z);
            } else {
                arrive(cur, tot, true, t, meta.z);   // the row begins in this tile
            }
        }
        __syncthreads();   // stage s and the scan scratch are free for reuse
    }

    if (failed) {
        if (tid == 0) {
            atomicOr(dev_status, kDevErrTimeout);
            // Let every bulk copy this block issued land before the block retires.
            const int hi = (i + STAGES) < mine ? (i + STAGES) : mine;
            for (int j = i; j < hi; ++j) (void)mbar_wait_bounded(&s_bar[j % STAGES], (j / STAGES) & 1);
        }
        __syncthreads();
    }
    epi.finish(est);
}

// Rows without entries see the value 0 (empty-row list, or every row when nnz == 0).
template <class Epi, typename AccT>
__global__ void __launch_bounds__(256)
    empty_rows_kernel(int count, const int* __restrict__ list, const Epi epi) {
    typename Epi::State est;
    epi.init(est);
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
        epi.apply(est, list ? list[k] : k, AccT(0));
    epi.finish(est);
}

// ---------------------------------------------------------------------------
// Block-level reduction helpers used by epilogues' finish().
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block max of non-negative values -> atomic max into *out (NaN-free inputs).
__device__ __forceinline__ void block_max_to(double v, double* out) {
    __shared__ double s_red[32];
    v = warp_max(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) s_red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double w = lane < nw ? s_red[lane] : 0.0;
        w = warp_max(w);
        if (lane == 0) atomic_max_nonneg(out, w);
    }
    __syncthreads();
}

}  // namespace pb
