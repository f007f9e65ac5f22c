// spmv.cuh — nnz-balanced ("merge-path") CSR SpMV for sm_100a with a fused
// per-row epilogue.
//
// Replaces the reference's csr_spmv_kernel (src/gpu/pdhg_kernels.cuh:24-37,
// one thread per row) and csr_spmv_t_kernel (:42-54, atomic scatter).  The
// transpose product is run by the same kernel over a stored transpose, so
// both products are gathers and both are deterministic run to run.
//
// Work decomposition
//   The nnz array is cut into tiles of T = BLOCK*IPT consecutive non-zeros.
//   A persistent grid (a multiple of the SM count) walks the tiles with a
//   static stride.  One elected thread streams each tile's col/val slabs into
//   a STAGES-deep shared-memory ring with 1-D TMA bulk copies
//   (cp.async.bulk ... mbarrier::complete_tx, L2 evict_first) while the
//   block works on earlier tiles.  Every thread owns IPT consecutive
//   non-zeros of the tile; it gathers x[col], multiplies, and walks the row
//   boundaries (row_ptr slice staged in shared memory).  Rows that end inside
//   the thread are finished on the spot; the rest are combined by a
//   segmented block scan (warp shuffles + one shared-memory pass), and rows
//   that cross a tile boundary by a "last arriver" rule: each tile holding a
//   piece of such a row stores its partial in carry[], fences, and bumps the
//   row's counter; the tile that brings the counter to the number of pieces
//   adds the partials in tile order and runs the epilogue.  No thread ever
//   waits on another block, and the summation order is fixed, so results
//   are bit-identical between runs.
//
// Row ownership: row r is finished by the thread whose item range (k0, k1]
// contains row_ptr[r+1] (row 0..: thread 0 of tile 0 also owns rows ending at
// 0).  Empty rows are therefore covered without a separate pass.  The device
// row_ptr carries one extra entry row_ptr[rows+1] = nnz_pad: the padding
// items [nnz, nnz_pad) (col 0, val 0) belong to a virtual row `rows` that is
// never emitted.
#pragma once

#include "common.cuh"

namespace pb {

// Device view of one CSR operand in the tiled layout.
struct CsrView {
    int rows = 0, cols = 0;
    int nnz = 0, nnz_pad = 0, num_tiles = 0;
    const int* row_ptr = nullptr;    // rows + 2 entries
    const int* col = nullptr;        // nnz_pad
    const float* val = nullptr;      // nnz_pad, value rounded to FP32
    const float* val_lo = nullptr;   // nnz_pad, FP32 of (value - val) or null
    const int* tile_row = nullptr;   // num_tiles + 1
    void* carry = nullptr;           // 2 * num_tiles accumulators (double-sized slots)
    int* counter = nullptr;          // num_tiles, zero between launches
};

// Default tile geometry: 256 threads x 8 non-zeros = 2048 non-zeros per tile.
constexpr int kSpmvBlock = 256;
constexpr int kSpmvIpt = 8;
constexpr int kSpmvTile = kSpmvBlock * kSpmvIpt;
constexpr int kSpmvStages = 4;

template <int BLOCK, int IPT, int STAGES, bool kLo, typename AccT>
struct SpmvSmemLayout {
    static constexpr int T = BLOCK * IPT;
    static constexpr int NW = BLOCK / 32;
    static constexpr int RP_CAP = T + 8;   // row_ptr slice capacity (entries)
    static constexpr int kArrays = kLo ? 3 : 2;
    static constexpr size_t off_col = 0;
    static constexpr size_t off_val = off_col + size_t(STAGES) * T * 4;
    static constexpr size_t off_lo = off_val + size_t(STAGES) * T * 4;
    static constexpr size_t off_rp = off_val + size_t(STAGES) * T * 4 * (kArrays - 1);
    static constexpr size_t off_bar = off_rp + size_t(RP_CAP) * 4;
    static constexpr size_t off_wrow = off_bar + size_t(STAGES) * 8;
    static constexpr size_t off_wval = off_wrow + size_t(NW) * 4 + 8;
    static constexpr size_t bytes = ((off_wval + size_t(NW) * sizeof(AccT)) + 127) / 128 * 128;
    static_assert(RP_CAP % 2 == 0, "mbarriers need 8-byte alignment");
};

// Epilogue concept:
//   struct Epi {
//     struct State {...};                         // per-thread state
//     __device__ void init(State&) const;
//     __device__ void apply(State&, int row, AccT value) const;   // row complete
//     __device__ void finish(State&) const;       // called once by every thread at exit
//   };

template <class Epi, typename AccT, typename XT, bool kLo, int BLOCK, int IPT, int STAGES>
__global__ void __launch_bounds__(BLOCK)
    spmv_merge_kernel(const CsrView A, const XT* __restrict__ x, const Epi epi,
                      int* __restrict__ dev_status) {
    using L = SpmvSmemLayout<BLOCK, IPT, STAGES, kLo, AccT>;
    constexpr int T = L::T;
    constexpr int NW = L::NW;
    static_assert(IPT % 4 == 0, "IPT must allow 16-byte shared-memory vector reads");

    extern __shared__ __align__(128) unsigned char smem[];
    int* s_col = reinterpret_cast<int*>(smem + L::off_col);
    float* s_val = reinterpret_cast<float*>(smem + L::off_val);
    float* s_lo = reinterpret_cast<float*>(smem + L::off_lo);
    int* s_rp = reinterpret_cast<int*>(smem + L::off_rp);
    uint64_t* s_bar = reinterpret_cast<uint64_t*>(smem + L::off_bar);
    int* s_wrow = reinterpret_cast<int*>(smem + L::off_wrow);
    AccT* s_wval = reinterpret_cast<AccT*>(smem + L::off_wval);

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int m = A.rows;
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
        mbar_arrive_expect_tx(&s_bar[s], unsigned(T) * 4u * L::kArrays);
        tma_bulk_g2s(s_col + s * T, A.col + off, T * 4, &s_bar[s], policy);
        tma_bulk_g2s(s_val + s * T, A.val + off, T * 4, &s_bar[s], policy);
        if constexpr (kLo) tma_bulk_g2s(s_lo + s * T, A.val_lo + off, T * 4, &s_bar[s], policy);
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

        const int r_lo = A.tile_row[t];
        const int r_hi = A.tile_row[t + 1];
        const int cnt = r_hi - r_lo + 2;
        const bool rp_smem = cnt <= L::RP_CAP;
        if (rp_smem) {
            for (int j = tid; j < cnt; j += BLOCK) s_rp[j] = A.row_ptr[r_lo + j];
        }
        const int* rpb = rp_smem ? (s_rp - r_lo) : A.row_ptr;   // rpb[r] == row_ptr[r]

        const bool ok = mbar_wait_bounded(&s_bar[s], parity);
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }

        const int tile_base = t * T;
        const int tile_end = tile_base + T;
        const int k0 = tile_base + tid * IPT;
        const int k1 = k0 + IPT;

        // ---- products: IPT independent gathers in flight per thread ----
        AccT p[IPT];
        {
            const int* sc = s_col + s * T + tid * IPT;
            const float* sv = s_val + s * T + tid * IPT;
#pragma unroll
            for (int j = 0; j < IPT; j += 4) {
                const int4 c4 = *reinterpret_cast<const int4*>(sc + j);
                const float4 v4 = *reinterpret_cast<const float4*>(sv + j);
                const int cc[4] = {c4.x, c4.y, c4.z, c4.w};
                const float vv[4] = {v4.x, v4.y, v4.z, v4.w};
                float ll[4] = {0.f, 0.f, 0.f, 0.f};
                if constexpr (kLo) {
                    const float4 l4 = *reinterpret_cast<const float4*>(s_lo + s * T + tid * IPT + j);
                    ll[0] = l4.x; ll[1] = l4.y; ll[2] = l4.z; ll[3] = l4.w;
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    unsigned ci = static_cast<unsigned>(cc[q]);
                    ci = ci < last_col ? ci : last_col;   // cheap guard: never gather out of bounds
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

        // ---- first row whose end lies beyond k0 ----
        int r;
        {
            int lo = r_lo, hi = r_hi;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (rpb[mid + 1] > k0) hi = mid; else lo = mid + 1;
            }
            r = (t == 0 && tid == 0) ? 0 : lo;
        }

        // ---- walk items and row boundaries ----
        AccT acc = AccT(0);
        int nemit = 0;
        int head_row = -1;
        AccT head_acc = AccT(0);
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            const int k = k0 + j;
            while (r < m && rpb[r + 1] <= k) {
                if (nemit == 0 && rpb[r] < k0) { head_row = r; head_acc = acc; }
                else epi.apply(est, r, acc);
                ++nemit; acc = AccT(0); ++r;
            }
            acc += p[j];
        }
        while (r < m && rpb[r + 1] <= k1) {
            if (nemit == 0 && rpb[r] < k0) { head_row = r; head_acc = acc; }
            else epi.apply(est, r, acc);
            ++nemit; acc = AccT(0); ++r;
        }

        // ---- segmented block scan of (tail row, tail partial) ----
        int krow = r;
        AccT kval = acc;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int ro = __shfl_up_sync(0xffffffffu, krow, d);
            const AccT vo = __shfl_up_sync(0xffffffffu, kval, d);
            if (lane >= d && ro == krow) kval += vo;
        }
        if (lane == 31) { s_wrow[warp] = krow; s_wval[warp] = kval; }
        __syncthreads();
        int prow = -1;
        AccT pval = AccT(0);
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            if (w < warp) {
                const int rw = s_wrow[w];
                const AccT vw = s_wval[w];
                if (rw == prow) pval += vw; else { prow = rw; pval = vw; }
            }
        }
        if (krow == prow) kval += pval;   // block-inclusive value of this thread
        int erow = __shfl_up_sync(0xffffffffu, krow, 1);
        AccT eval = __shfl_up_sync(0xffffffffu, kval, 1);
        if (lane == 0) { erow = prow; eval = pval; }

        auto cross_tile = [&](int row, AccT v, bool is_tail) {
            carry[2 * t + (is_tail ? 1 : 0)] = v;
            __threadfence();
            const int t0 = rpb[row] / T;
            const int t1 = (rpb[row + 1] - 1) / T;
            const int old = atomicAdd(&A.counter[t0], 1);
            if (old == t1 - t0) {
                __threadfence();
                AccT sum = ld_cg(&carry[2 * t0 + 1]);
                for (int tt = t0 + 1; tt <= t1; ++tt) sum += ld_cg(&carry[2 * tt]);
                A.counter[t0] = 0;
                epi.apply(est, row, sum);
            }
        };

        if (head_row >= 0) {
            const AccT tot = head_acc + (erow == head_row ? eval : AccT(0));
            if (rpb[head_row] >= tile_base) epi.apply(est, head_row, tot);
            else cross_tile(head_row, tot, false);
        }
        // The tile's last row continues into the next tile: a piece of it
        // lies in this tile only when the row starts before tile_end (a row
        // starting exactly on the boundary belongs wholly to later tiles).
        if (tid == BLOCK - 1 && krow < m && rpb[krow] < tile_end && rpb[krow + 1] > tile_end) {
            cross_tile(krow, kval, rpb[krow] >= tile_base);
        }
        __syncthreads();   // stage s, s_rp and s_w* free for reuse
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

// Rows of an operand without any non-zero (nnz == 0): every row sees 0.
template <class Epi, typename AccT>
__global__ void __launch_bounds__(256) zero_rows_kernel(int rows, const Epi epi) {
    typename Epi::State est;
    epi.init(est);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
        epi.apply(est, r, AccT(0));
    epi.finish(est);
}

// ---------------------------------------------------------------------------
// Block-level reduction helper used by epilogues' finish().
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
