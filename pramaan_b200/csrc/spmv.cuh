// spmv.cuh — nnz-balanced ("merge-path") CSR SpMV for sm_100a with a fused
// per-row epilogue.
//
// Replaces the reference's csr_spmv_kernel (src/gpu/pdhg_kernels.cuh:24-37,
// one thread per row) and csr_spmv_t_kernel (:42-54, atomic scatter).  The
// transpose product is run by the same kernel over a stored transpose, so
// both products are gathers and both are deterministic run to run.
//
// Tiled operand format (built once per matrix, see csr_device.cu)
//   The non-zeros are cut into tiles of TW = 32*IPT consecutive entries, one
//   tile per warp at a time.  Each tile is ONE contiguous record, so a single
//   ~4 KB bulk copy moves it (copies of 2 KB or less stream at well under
//   half of HBM bandwidth on B200; 4 KB and up reach it):
//     col   int32[TW]     column indices  (lane-interleaved, see tile_slot)
//     val   fp32 [TW]     values (FP32-rounded, same order)
//     flags u32 [TW/32]   bit q set <=> entry q starts a row
//     meta  int4          {first_row, tail_continues, 0, 0}
//   The FP32 remainders val_lo (value - val), when present, stay in a flat
//   array and travel in a second copy, only for the FP64 products.
//   Empty rows are compacted out (an optional row_map gives the original row
//   of every compacted row) and the padding after the last entry forms a
//   virtual row that is never emitted, so row ids follow from the bitmap
//   alone: row(q) = first_row + #starts in (0, q].  The kernel never reads
//   row_ptr.
//
// Hot gather targets
//   When a few x entries take a large share of the gathers (the transpose of
//   an LP with power-law row lengths: every entry of a long row of A gathers
//   the same y), the operand lists them as hot slots (hot_idx[slot] = target)
//   and its records hold ~slot (a negative index) for those entries.  The
//   FP32 kernels copy the hot targets into shared memory once per block and
//   read them from there, so only the cold gathers reach L2; other kernels
//   resolve ~slot through hot_idx.  The value gathered, and so every sum, is
//   the same either way.
//
// Local gathers
//   The default gathers (ld.global.cg) skip L1: on a random pattern caching
//   them only evicts lines other warps wait on.  When an operand's columns are
//   local (banded and multi-period structures), ld.global.ca lets neighbouring
//   rows reuse the lines in L1; the launch autotuner times both and records
//   the faster in the operand (gather_l1).
//
// What bounds it
//   On a random sparsity pattern every entry costs one 4-byte gather of x
//   from L2, and B200 serves random gathers at about one sector request per
//   clock per SM, whatever the cache operator: 279 G gathers/s measured by
//   gather_ceiling_kernel (ceiling.cu), with the L1-to-crossbar request path
//   97 % busy.  The matrix stream itself needs well under half of HBM
//   bandwidth at that rate (the Ax̄ product of a 108 M-entry power-law LP runs
//   at 0.84 of the gather rate).  Outstanding gather misses occupy L1 lines,
//   so the plain kernel runs with a shared-memory carve-out sized for 3 blocks
//   per SM (leaving ~100 KB of L1) rather than the largest carve-out: with the
//   L1 squeezed to ~40 KB the same kernel runs at half the gather rate.  When
//   the gathers are local (they hit L1) the product is latency-bound instead,
//   and the dense variants (kStageAlias: finished rows staged over the tile's
//   own slots, 4-5 blocks per SM) hide more of that latency.
//
// Schedule (spmv_warp_kernel)
//   A persistent grid walks the tiles; every warp owns a private STAGES-deep
//   shared-memory ring that its lane 0 fills with 1-D TMA bulk copies
//   (cp.async.bulk ... mbarrier::complete_tx, L2 evict_first), so warps never
//   wait on each other: there is no block barrier in the main loop.  Each
//   lane owns IPT consecutive entries, read as conflict-free 16-byte chunks:
//   it issues its IPT x gathers first, row ids come from popcounts of the
//   bitmap (bit-plane ballots for the prefix), the epilogue's
//   vectors for the tile's finished rows are prefetched into L2, products
//   are accumulated with FMAs, and a segmented warp scan carries open-row
//   partial sums across lanes (shuffles for the sums, one ballot for where
//   rows end).  The rows finished in the tile are
//   consecutive, so their sums are staged in a per-warp shared buffer and the
//   epilogue then runs converged, one row per lane, with coalesced loads and
//   stores.  A row that crosses tiles leaves one partial per tile in carry[]
//   (head piece: the tile holds its end or a middle part; tail piece: it
//   begins in the tile).
//
// Completion (spmv_fixup_kernel, launched right after on the same stream)
//   For every crossing row the fixup adds its pieces in tile order and runs
//   the epilogue; it also gives every empty row the value 0.  All sums have a
//   fixed order, so results are bit-identical between runs, and no thread
//   ever waits on another block.
#pragma once

#include "common.cuh"

namespace pb {

constexpr int kSpmvIpt = 16;                 // entries per lane
constexpr int kSpmvTile = 32 * kSpmvIpt;     // entries per warp-tile (format unit)

// Slot of tile-local entry q in a record's column and value arrays (and in
// the tile's val_lo slab).  Lane l owns entries IPT*l .. IPT*l + IPT-1 and
// reads them as 16-byte chunks; chunk k of lane l is stored at chunk index
// k*32 + l, so each chunk read of a warp is 512 contiguous bytes of shared
// memory (4 wavefronts) instead of 32 reads at a 64-byte stride (16).
__host__ __device__ constexpr int tile_slot(int q) {
    return (((q % kSpmvIpt) / 4) * 32 + q / kSpmvIpt) * 4 + (q % 4);
}

static_assert(tile_slot(0) == 0 && tile_slot(4) == 128 && tile_slot(16) == 4 && tile_slot(511) == 511,
              "tile_slot layout");

// Byte layout of one tile record.
struct TileRec {
    static constexpr int TW = kSpmvTile;
    static constexpr int FW = TW / 32;
    static constexpr size_t off_col = 0;
    static constexpr size_t off_val = size_t(TW) * 4;
    static constexpr size_t off_flags = size_t(TW) * 8;
    static constexpr size_t off_meta = off_flags + size_t(FW) * 4;
    static constexpr size_t bytes = off_meta + 16;
    static_assert(bytes % 16 == 0, "tile records must be 16-byte multiples");
};

// Device view of one CSR operand in the tiled format.
struct CsrView {
    int rows = 0;          // original rows (epilogue index space)
    int cols = 0;
    int nnz = 0, nnz_pad = 0, num_tiles = 0;
    int rows_c = 0;        // non-empty (compacted) rows
    int num_empty = 0;     // rows without entries
    int num_cross = 0;     // rows spanning more than one tile
    int blocks_per_sm = 0; // grid = blocks_per_sm x SMs (0: library default)
    const unsigned char* rec = nullptr;   // num_tiles tile records (TileRec)
    const float* val_lo = nullptr;        // nnz_pad or null
    const int* row_map = nullptr;     // rows_c (null: identity)
    const int* empty_rows = nullptr;  // num_empty
    const int4* cross = nullptr;      // num_cross: {original row, first tile, tiles, 0}
    void* carry = nullptr;            // 2 * num_tiles accumulators (8-byte slots)
    int hot = 0;                      // hot gather slots (records hold ~slot for them)
    const int* hot_idx = nullptr;     // hot: gather target of every slot
    int gather_l1 = 0;                // gathers cached in L1 (operands without hot slots)
    int l2_resident = 0;              // records fit in L2 with the iteration's vectors: keep them
};

// Gather modes of the product kernel.
constexpr int kGatherL2 = 0;       // ld.global.cg
constexpr int kGatherHot = 1;      // ~slot from the block's shared copy, the rest ld.global.cg
constexpr int kGatherHotIdx = 2;   // ~slot resolved through hot_idx
constexpr int kGatherL1 = 3;       // ld.global.ca

// Predicated ld.global.cg: the load is issued only when `pred` holds, so hot
// lanes send no request at all (pointing them all at one address instead
// concentrates the requests of every SM on one L2 slice: measured 2x slower).
// The address must be valid either way; callers pass an in-range one.  Not
// volatile: the compiler may schedule it like an ordinary load.
__device__ __forceinline__ float ldcg_if(const float* p, bool pred) {
    float v = 0.f;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q ld.global.cg.f32 %0, [%1];\n\t}"
        : "+f"(v) : "l"(p), "r"(int(pred)));
    return v;
}
__device__ __forceinline__ double ldcg_if(const double* p, bool pred) {
    double v = 0.0;
    asm("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q ld.global.cg.f64 %0, [%1];\n\t}"
        : "+d"(v) : "l"(p), "r"(int(pred)));
    return v;
}

// Gather of entry index c in mode kG (hs: the block's shared copy of the hot
// targets).  Every address formed is in range whichever way the selects go.
template <int kG, typename XT>
__device__ __forceinline__ XT spmv_gather(const XT* __restrict__ x, const XT* hs, const CsrView& A, int c) {
    if constexpr (kG == kGatherHot) {
        const bool cold = c >= 0;
        const XT g = ldcg_if(x + (cold ? c : 0), cold);
        const XT h = hs[cold ? 0 : ~c];
        return cold ? g : h;
    } else if constexpr (kG == kGatherHotIdx) {
        const int t = __ldg(A.hot_idx + (c >= 0 ? 0 : ~c));
        return __ldcg(x + (c >= 0 ? c : t));
    } else if constexpr (kG == kGatherL1) {
        return __ldca(x + c);
    } else {
        return __ldcg(x + c);
    }
}

// kAlias: the finished-row values of a tile are staged over the tile's own
// column / value slots (every lane has moved those to registers by then), so
// a warp needs no shared memory beyond its ring.  Used by the hot-slot
// kernel, whose block also holds the hot copy: the saving buys it warps.
template <int WARPS, int STAGES, bool kLo, typename AccT, bool kAlias = false>
struct SpmvSmemLayout {
    static constexpr int TW = kSpmvTile;
    static constexpr int FW = TileRec::FW;
    static constexpr size_t off_val = TileRec::off_val;
    static constexpr size_t off_flags = TileRec::off_flags;
    static constexpr size_t off_meta = TileRec::off_meta;
    static constexpr size_t off_lo = TileRec::bytes;                         // kLo only
    static constexpr size_t stage_bytes = TileRec::bytes + (kLo ? size_t(TW) * 4 : 0);
    static constexpr size_t off_fin = size_t(STAGES) * stage_bytes;        // finished-row values (no alias)
    static constexpr size_t warp_bytes =
        kAlias ? (off_fin + 15) / 16 * 16 : (off_fin + size_t(TW) * sizeof(AccT) + 15) / 16 * 16;
    static_assert(!kAlias || size_t(TW) * sizeof(AccT) <= off_flags,
                  "staged row values must fit in the column / value slots");
    static constexpr size_t off_bar = size_t(WARPS) * warp_bytes;
    static constexpr size_t bytes = ((off_bar + size_t(WARPS) * STAGES * 8) + 127) / 128 * 128;
    static constexpr unsigned tx_bytes = unsigned(stage_bytes);
    static_assert(stage_bytes % 16 == 0, "TMA copies must be 16-byte multiples");
};

// Epilogue concept:
//   struct Epi {
//     struct State {...};                                  // per-thread state
//     __device__ void init(State&) const;
//     __device__ void prefetch(int row) const;             // L2 prefetch of row data
//     __device__ void apply(State&, int row, AccT value) const;   // row complete
//     __device__ void finish(State&, int channel) const;   // once by every thread at exit
//                                                          // (channel 0: main kernel, 1: fixup)
//   };

// Epilogues that split apply() into load(row) -> In and store(State&, row,
// In, value) declare `static constexpr bool kSplit = true`; the tile loop
// then loads kEpiPass rows per lane ahead of their updates.
template <class Epi, class = void>
struct EpiSplit { static constexpr bool value = false; };
template <class Epi>
struct EpiSplit<Epi, decltype(void(Epi::kSplit))> { static constexpr bool value = Epi::kSplit; };
constexpr int kEpiPass = 4;

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// One product over the tiles of A, run by every warp of the grid (warp w of
// block b takes tiles b*WARPS + w, + gridDim.x*WARPS, ...).  `used` counts the
// tiles this warp's ring consumed in earlier products of the same kernel (0 and
// `init_bars` for the first), so the ring's mbarrier phases carry over from one
// product to the next.  `ready()` is called by every thread after the first
// bulk copies are issued and before anything but the tile records is read or
// written: a grid dependency wait, or a grid barrier in a multi-product
// kernel; it returns false to abandon the product.  Returns false when a wait
// gave up (the status word records it).
// kG: gather mode (spmv_gather).  With kGatherHot the block's copy of the
// hot targets sits after the rings (shared-memory offset L::bytes, A.hot
// values of XT).
// kStageAlias: stage the finished rows over the tile's column / value slots
// in any gather mode (the hot-slot mode always does), so a warp needs only its
// ring and more warps fit on an SM.
template <class Epi, typename AccT, typename XT, bool kLo, bool kRowMap, int WARPS, int STAGES, int kG = kGatherL2,
          bool kStageAlias = false, class Ready>
__device__ __forceinline__ bool spmv_tiles(const CsrView& A, const XT* __restrict__ x, const Epi& epi,
                                           int* __restrict__ dev_status, unsigned char* smem, uint32_t& used,
                                           bool init_bars, Ready&& ready) {
    constexpr bool kAlias = kG == kGatherHot || kStageAlias;
    using L = SpmvSmemLayout<WARPS, STAGES, kLo, AccT, kAlias>;
    constexpr int IPT = kSpmvIpt;
    constexpr int TW = L::TW;
    constexpr int FW = L::FW;
    constexpr unsigned kMask = (IPT == 32) ? 0xffffffffu : ((1u << IPT) - 1u);

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    unsigned char* ring = smem + size_t(warp) * L::warp_bytes;
    // staged row values: a per-warp buffer, or (aliased) the current stage, set per tile
    AccT* fin = kAlias ? nullptr : reinterpret_cast<AccT*>(ring + L::off_fin);
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + L::off_bar) + warp * STAGES;

    const int rows_c = A.rows_c;

    typename Epi::State est;
    epi.init(est);

    const int nt = A.num_tiles;
    const int gw = blockIdx.x * WARPS + warp;
    const int stride = gridDim.x * WARPS;
    const int mine = gw < nt ? (nt - gw + stride - 1) / stride : 0;

    uint64_t policy = 0;
    if (lane == 0) {
        if (init_bars) {
            for (int s = 0; s < STAGES; ++s) mbar_init(&bar[s], 1);
            fence_mbar_init();
        }
        // Records of an operand that fits in L2 (with the other operand and the
        // vectors) stay there for the next launch; the others stream through.
        policy = A.l2_resident ? l2_policy_evict_last() : l2_policy_evict_first();
    }
    __syncwarp();

    auto issue = [&](int i) {
        const int t = gw + i * stride;
        const int s = int((used + uint32_t(i)) % STAGES);
        unsigned char* st = ring + size_t(s) * L::stage_bytes;
        const size_t off = size_t(t) * TW;
        mbar_arrive_expect_tx(&bar[s], L::tx_bytes);
        tma_bulk_g2s(st, A.rec + size_t(t) * TileRec::bytes, unsigned(TileRec::bytes), &bar[s], policy);
        if constexpr (kLo) tma_bulk_g2s(st + L::off_lo, A.val_lo + off, TW * 4, &bar[s], policy);
    };

    if (lane == 0) {
        fence_proxy_async_smem();
        const int pre = mine < STAGES ? mine : STAGES;
        for (int i = 0; i < pre; ++i) issue(i);
    }
    // The tile records are never written while products run, so the first
    // copies above may overlap earlier work; x, the epilogue's vectors and
    // carry[] are touched only once ready() has returned.
    bool failed = !ready();

    XT* hs = reinterpret_cast<XT*>(smem + L::bytes);
    if constexpr (kG == kGatherHot) {
        __syncthreads();   // an earlier product of the same kernel may still read the copy
        const int H = A.hot;
        constexpr int U = 8;
        for (int k0 = threadIdx.x; k0 < H; k0 += WARPS * 32 * U) {
            XT v[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + u * WARPS * 32;
                v[u] = k < H ? __ldcg(x + __ldg(A.hot_idx + k)) : XT(0);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int k = k0 + u * WARPS * 32;
                if (k < H) hs[k] = v[u];
            }
        }
        __syncthreads();
    }

    AccT* carry = reinterpret_cast<AccT*>(A.carry);
    int i = 0;
    for (; i < mine && !failed; ++i) {
        const int t = gw + i * stride;
        const uint32_t u = used + uint32_t(i);
        const int s = int(u % STAGES);
        const uint32_t parity = (u / STAGES) & 1u;
        const bool ok = mbar_wait_bounded(&bar[s], parity);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        const unsigned char* st = ring + size_t(s) * L::stage_bytes;
        const int4* scol4 = reinterpret_cast<const int4*>(st);                  // tile_slot order
        const float4* sval4 = reinterpret_cast<const float4*>(st + L::off_val);
        const float4* slo4 = reinterpret_cast<const float4*>(st + L::off_lo);
        const uint32_t* fl = reinterpret_cast<const uint32_t*>(st + L::off_flags);
        const int4 meta = *reinterpret_cast<const int4*>(st + L::off_meta);
        const int q0 = lane * IPT;   // tile-local index of my first entry

        // ---- gather x for my entries first: IPT independent loads in flight ----
        XT xv[IPT];
        float vv[IPT];
        float ll[IPT];
#pragma unroll
        for (int j = 0; j < IPT; j += 4) {
            const int4 c4 = scol4[(j / 4) * 32 + lane];    // my entries q0 + j .. q0 + j + 3
            const float4 v4 = sval4[(j / 4) * 32 + lane];
            // ld.global.cg: the gathers are served by L2; caching them in L1
            // only evicts lines other warps are waiting on.
            xv[j] = spmv_gather<kG>(x, hs, A, c4.x); xv[j + 1] = spmv_gather<kG>(x, hs, A, c4.y);
            xv[j + 2] = spmv_gather<kG>(x, hs, A, c4.z); xv[j + 3] = spmv_gather<kG>(x, hs, A, c4.w);
            vv[j] = v4.x; vv[j + 1] = v4.y; vv[j + 2] = v4.z; vv[j + 3] = v4.w;
            if constexpr (kLo) {
                const float4 l4 = slo4[(j / 4) * 32 + lane];
                ll[j] = l4.x; ll[j + 1] = l4.y; ll[j + 2] = l4.z; ll[j + 3] = l4.w;
            }
        }
        if constexpr (kAlias) {
            // every lane holds its columns and values now: the slots take the staged rows
            __syncwarp();
            fin = reinterpret_cast<AccT*>(const_cast<unsigned char*>(st));
        }

        // ---- row-start bits of my entries and of the entry after them ----
        const uint32_t my = (fl[q0 >> 5] >> (q0 & 31)) & kMask;
        uint32_t next_start;
        if (lane == 31) next_start = meta.y ? 0u : 1u;
        else next_start = (fl[(q0 + IPT) >> 5] >> ((q0 + IPT) & 31)) & 1u;
        const uint32_t ends = (my >> 1) | (next_start << (IPT - 1));   // bit j: entry j ends a row
        const int s0 = int(fl[0] & 1u);                                 // tile's first entry starts a row

        // ---- row ids: first_row + #starts in (0, q] ----
        // Each lane's start count (0..16) in five bit-planes: one ballot per
        // plane gives the exclusive prefix and the total without shuffles.
        const int cnt = __popc(my);
        int excl = 0, starts_total = 0;
        const unsigned below = (1u << lane) - 1u;
#pragma unroll
        for (int b = 0; b < 5; ++b) {
            const unsigned plane = __ballot_sync(0xffffffffu, (cnt >> b) & 1);
            excl += __popc(plane & below) << b;
            starts_total += __popc(plane) << b;
        }
        const int row0 = meta.x + excl + int(my & 1u) - s0;
        const bool head_before = (my & 1u) == 0;   // my first row began before my first entry

        // Rows finished in this tile are meta.x .. meta.x + ends_total - 1.  When
        // the tile's first row began in an earlier tile, its finish here is a
        // carry piece, so the staged list starts one row later.
        const int ends_total = starts_total - s0 + (meta.y ? 0 : 1);
        const int skip = (s0 == 0 && ends_total > 0) ? 1 : 0;
        const int base = meta.x + skip;
        int n_fin = ends_total - skip;
        if (n_fin > rows_c - base) n_fin = rows_c - base;   // virtual padding row
        if constexpr (!kRowMap) {
            for (int k = lane * 8; k < n_fin; k += 256) epi.prefetch(base + k);
        }

        // ---- walk my entries; stage the rows that end here ----
        // Without branches: the first row end closes the head row when that
        // row began before my first entry (head_bit); every other end stores
        // its row into the staging buffer at row0 - base + (ends before it),
        // a predicated store.  The sums are the same FMAs in the same order.
        const uint32_t head_bit = head_before ? (ends & (0u - ends)) : 0u;
        const bool head_pending = head_bit != 0u;
        AccT* const fin_row = fin + (row0 - base);
        AccT acc = AccT(0);
        AccT head_acc = AccT(0);
        int k_end = 0;
#pragma unroll
        for (int j = 0; j < IPT; ++j) {
            if constexpr (kLo) {
                acc = fma(static_cast<AccT>(vv[j]) + static_cast<AccT>(ll[j]), static_cast<AccT>(xv[j]), acc);
            } else {
                acc = fma(static_cast<AccT>(vv[j]), static_cast<AccT>(xv[j]), acc);
            }
            const bool e = (ends >> j) & 1u;
            const bool h = (head_bit >> j) & 1u;
            if (e && !h) fin_row[k_end] = acc;
            head_acc = h ? acc : head_acc;
            k_end += e ? 1 : 0;
            acc = e ? AccT(0) : acc;
        }
        const int nemit = k_end;
        const int cur = row0 + k_end;

        // ---- segmented warp scan of (row end seen, open partial) ----
        // Before the step of distance d, lane i's partial covers lanes
        // (i-d, i]; it takes lane i-d's only when no lane in that window
        // ended a row, read from one ballot of the row ends.
        const unsigned ended = __ballot_sync(0xffffffffu, nemit > 0) & (lane == 31 ? 0xffffffffu : ((2u << lane) - 1u));
        AccT v = acc;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const AccT vo = __shfl_up_sync(0xffffffffu, v, d);
            const int lo = lane - d + 1 > 0 ? lane - d + 1 : 0;
            if (lane >= d && (ended >> lo) == 0u) v += vo;
        }
        AccT carry_in = __shfl_up_sync(0xffffffffu, v, 1);   // partial of the row open at q0
        if (lane == 0) carry_in = AccT(0);

        if (head_pending) {
            const AccT tot = head_acc + carry_in;
            if (row0 == meta.x && s0 == 0) carry[2 * t] = tot;   // last piece of a crossing row
            else fin[row0 - base] = tot;
        }
        if (lane == 31 && meta.y) {   // the tile's last row continues into the next tile
            const AccT tot = nemit > 0 ? acc : carry_in + acc;
            if (cur == meta.x && s0 == 0) carry[2 * t] = tot;    // middle piece
            else carry[2 * t + 1] = tot;                         // first piece
        }
        __syncwarp();

        // ---- epilogue over the finished rows, one row per lane (coalesced) ----
        if constexpr (EpiSplit<Epi>::value) {
            // Epilogues with a separate load step: the inputs of kEpiPass rows
            // per lane are loaded before any of them is updated, so the loads
            // of a tile with many short rows overlap instead of running one
            // round trip per 32 rows.
            constexpr int U = kEpiPass;
            for (int k0 = lane; k0 < n_fin; k0 += 32 * U) {
                typename Epi::In in[U];
                int row[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int k = k0 + 32 * u;
                    row[u] = k < n_fin ? (kRowMap ? A.row_map[base + k] : base + k) : -1;
                    if (row[u] >= 0) in[u] = epi.load(row[u]);
                }
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (row[u] >= 0) epi.store(est, row[u], in[u], fin[k0 + 32 * u]);
            }
        } else {
            for (int k = lane; k < n_fin; k += 32) {
                const int rc = base + k;
                epi.apply(est, kRowMap ? A.row_map[rc] : rc, fin[k]);
            }
        }
        __syncwarp();   // stage s and the staged values are free for reuse
        if (lane == 0 && i + STAGES < mine) {
            fence_proxy_async_smem();
            issue(i + STAGES);
        }
    }

    if (failed) {
        if (lane == 0) {
            atomicOr(dev_status, kDevErrTimeout);
            // Let every bulk copy this warp issued land before it retires.
            const int hi = (i + STAGES) < mine ? (i + STAGES) : mine;
            for (int j = i; j < hi; ++j) {
                const uint32_t u = used + uint32_t(j);
                (void)mbar_wait_bounded(&bar[u % STAGES], (u / STAGES) & 1u);
            }
        }
        __syncwarp();
    }
    used += uint32_t(mine);
    epi.finish(est, 0);
    return !failed;
}

template <class Epi, typename AccT, typename XT, bool kLo, bool kRowMap, int WARPS, int STAGES, int kG = kGatherL2,
          bool kStageAlias = false>
__global__ void __launch_bounds__(WARPS * 32, (sizeof(AccT) == 4 ? 5 : 4) * 4 / WARPS > 0
                                                  ? (sizeof(AccT) == 4 ? 5 : 4) * 4 / WARPS : 1)
    spmv_warp_kernel(const CsrView A, const XT* __restrict__ x, const Epi epi,
                     int* __restrict__ dev_status) {
    extern __shared__ __align__(128) unsigned char smem[];
    uint32_t used = 0;
    spmv_tiles<Epi, AccT, XT, kLo, kRowMap, WARPS, STAGES, kG, kStageAlias>(A, x, epi, dev_status, smem, used, true, [] {
        grid_dep_launch();
        grid_dep_wait();
        return true;
    });
}

// Finishes the rows that cross tiles (their pieces added in tile order) and
// gives every empty row the value 0.
// Thread `tid` of `nthreads` finishes its share of the crossing and empty
// rows.  The pieces are read past L1 (they are written by other warps, and a
// multi-product kernel reads them again after the next product).
template <class Epi, typename AccT>
__device__ __forceinline__ void spmv_fixup_rows(const CsrView& A, const Epi& epi, int tid, int nthreads) {
    typename Epi::State est;
    epi.init(est);
    const AccT* carry = reinterpret_cast<const AccT*>(A.carry);
    const int total = A.num_cross + A.num_empty;
    for (int k = tid; k < total; k += nthreads) {
        if (k < A.num_cross) {
            const int4 c = A.cross[k];   // {row, first tile, tiles, 0}
            AccT sum = __ldcg(carry + 2 * c.y + 1);
            for (int tt = c.y + 1; tt < c.y + c.z; ++tt) sum += __ldcg(carry + 2 * tt);
            epi.apply(est, c.x, sum);
        } else {
            epi.apply(est, A.empty_rows[k - A.num_cross], AccT(0));
        }
    }
    epi.finish(est, 1);
}

template <class Epi, typename AccT>
__global__ void __launch_bounds__(256)
    spmv_fixup_kernel(const CsrView A, const Epi epi) {
    grid_dep_launch();
    grid_dep_wait();
    spmv_fixup_rows<Epi, AccT>(A, epi, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
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
