// csr_device.cuh — device-resident CSR operands in the tiled format consumed
// by spmv_tile_kernel, plus the launch helpers.
//
// Layout in HBM (one operand; A and its stored transpose each get one):
//   row_ptr    int32 [rows + 1]        the CSR row pointer as given
//   rec        tile records [tiles]    per tile: col int32[512] (pad: 0),
//                                      val fp32[512] (FP32-rounded, pad: 0),
//                                      both lane-interleaved (tile_slot),
//                                      flags u32[16] (bit q: entry q starts a
//                                      non-empty row), meta int4
//                                      {first_row, tail_continues, 0, 0}
//   val_lo     fp32  [nnz_pad]         FP32(value - val), kept only when some
//                                      value is not exactly representable (entry
//                                      order while building, tile_slot order
//                                      once packed)
//   row_map    int32 [rows_c]          original row of each non-empty row (only
//                                      when empty rows exist)
//   empty_rows int32 [rows - rows_c]   rows without entries
//   cross      int4  [crossing rows]   {row, first tile, tiles, 0} per row spanning tiles
//   carry      f64   [2 * tiles]       per-tile partials of crossing rows (scratch)
//   hot_idx    int32 [hot]             gather target of every hot slot (records
//                                      hold ~slot for those entries; see spmv.cuh)
// nnz_pad is a multiple of the tile (512 entries); records are 4176 bytes and
// every array starts on a 256-byte boundary (cudaMalloc), so each record and
// each tile's val_lo slab is 16-byte aligned for the bulk copies.  While an
// operand is being built it is held as flat col / val / flags / meta arrays
// (what the transpose and the step-size pass read); pack() then interleaves
// them into the records and frees the flat copies.
#pragma once

#include <atomic>
#include <stdexcept>
#include <cstddef>
#include <functional>
#include <utility>
#include <vector>

#include "common.cuh"
#include "spmv.cuh"

namespace pb {

// ---------------------------------------------------------------------------
// Device allocations go through a process-wide cache (csr_device.cu): a
// solve allocates and frees several GB of operands and temporaries, and
// cudaMalloc / cudaFree of that much memory cost more per call than the
// transfers.  A freed block first waits for the device (cudaFree's
// synchronisation, which callers may rely on), then is kept for reuse by a
// later allocation of up to its size on the same device (best fit, at most
// twice the request); kDeviceCacheCap bytes at most are kept per device, and
// a failed cudaMalloc releases the cache and retries.
// ---------------------------------------------------------------------------
void* device_cache_alloc(size_t bytes);
void device_cache_free(void* p) noexcept;
// Frees the cached blocks of device `dev` (-1: every device).
void device_cache_release(int dev);

// RAII device buffer
template <typename T>
class DevBuf {
public:
    DevBuf() = default;
    explicit DevBuf(size_t n) { alloc(n); }
    ~DevBuf() { reset(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_) { o.p_ = nullptr; o.n_ = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { reset(); p_ = o.p_; n_ = o.n_; o.p_ = nullptr; o.n_ = 0; }
        return *this;
    }
    void alloc(size_t n) {
        reset();
        if (n == 0) return;
        p_ = static_cast<T*>(device_cache_alloc(n * sizeof(T)));
        n_ = n;
    }
    void reset() {
        if (p_) device_cache_free(p_);
        p_ = nullptr;
        n_ = 0;
    }
    T* get() const { return p_; }
    size_t size() const { return n_; }
    size_t bytes() const { return n_ * sizeof(T); }

private:
    T* p_ = nullptr;
    size_t n_ = 0;
};

class CsrDevice {
public:
    int rows = 0, cols = 0, nnz = 0, nnz_pad = 0, num_tiles = 0;
    int rows_c = 0, num_empty = 0, num_cross = 0;
    int tuned_blocks_per_sm = 0;   // set by the launch autotuner (0: default)
    int hot = 0;                   // hot gather slots
    int gather_l1 = 0;             // gathers cached in L1 (set by the launch autotuner)
    int l2_resident = 0;           // keep the records in L2 between launches (see mark_l2_resident)
    bool has_lo = false;
    bool packed = false;
    bool keep_flat = false;        // pack() keeps the flat col / val (FP32) arrays
                                   // for kernels that read the plain CSR
    DevBuf<int> row_ptr, col, row_map, empty_rows, hot_idx, hot_slot;
    DevBuf<float> val, val_lo;
    DevBuf<uint32_t> flags;
    DevBuf<int4> meta, cross;
    DevBuf<unsigned char> rec;
    DevBuf<double> carry;

    CsrView view(bool with_lo) const {
        CsrView v;
        v.rows = rows; v.cols = cols; v.nnz = nnz; v.nnz_pad = nnz_pad; v.num_tiles = num_tiles;
        v.rows_c = rows_c; v.num_empty = num_empty; v.num_cross = num_cross;
        v.blocks_per_sm = tuned_blocks_per_sm;
        if (!packed && num_tiles > 0) throw std::logic_error("CsrDevice::view before pack()");
        v.rec = rec.get();
        v.val_lo = (with_lo && has_lo) ? val_lo.get() : nullptr;
        v.row_map = row_map.get(); v.empty_rows = empty_rows.get();
        v.cross = cross.get(); v.carry = carry.get();
        v.hot = hot; v.hot_idx = hot_idx.get();
        v.gather_l1 = gather_l1;
        v.l2_resident = l2_resident;
        return v;
    }

    // Algorithmic bytes of one SpMV over this operand: 8 nnz (col + val) +
    // 4 (rows + 1) (row structure) + 4 cols (gathered vector, counted once) +
    // 4 rows (result).
    double spmv_bytes() const {
        return 8.0 * nnz + 4.0 * (rows + 1) + 4.0 * cols + 4.0 * rows;
    }

    // Allocates the padded arrays for the given shape.
    void allocate(int rows_, int cols_, int nnz_, bool lo);
    // Builds flags / meta / row compaction / crossing rows from row_ptr.
    void finalize(cudaStream_t st);
    // Interleaves col / val / flags / meta into tile records and frees them
    // (entries whose target has a hot slot get ~slot).
    void pack(cudaStream_t st);
    // Chooses the hot gather targets before pack(): `target_rp` is the row
    // pointer of the operand whose rows are this operand's gather targets
    // (A's for AT, AT's for A), so target i is gathered target_rp[i+1] -
    // target_rp[i] times.  A target gets a slot when it is gathered at least
    // kSpmvHotMinUses times per resident block of the hot kernel (each block
    // loads every slot once); the slots are kept only when they take at least
    // kSpmvHotMinShare of the non-zeros.  No-op for small operands.
    void select_hot(const int* target_rp, int num_targets, int dev, cudaStream_t st);
    size_t device_bytes() const {
        return row_ptr.bytes() + col.bytes() + row_map.bytes() + empty_rows.bytes() + hot_idx.bytes() +
               val.bytes() + val_lo.bytes() + flags.bytes() + meta.bytes() + cross.bytes() +
               rec.bytes() + carry.bytes();
    }
};

// Uploads a host CSR with FP64 values (reference ModelIR layout) and splits
// every value into FP32 hi + FP32 lo on the device.  `d_flag` receives a
// nonzero code when row_ptr is not monotone or a column index is out of range.
void csr_upload_f64(CsrDevice& A, int rows, int cols, int nnz, const int* h_row_ptr,
                    const int* h_col, const double* h_val, cudaStream_t st, int* d_flag);
// Uploads a host CSR with FP32 values (test-harness launchers).
void csr_upload_f32(CsrDevice& A, int rows, int cols, int nnz, const int* h_row_ptr,
                    const int* h_col, const float* h_val, cudaStream_t st, int* d_flag);
// Builds AT = transpose(A) on the device (stable: rows of AT list A's rows in
// increasing order, the order of the reference's counting-sort transpose,
// src/linalg/sparse_matrix.cpp:13-57).
void csr_transpose(const CsrDevice& A, CsrDevice& AT, cudaStream_t st);
// Hot gather slots for both operands of a product pair (before pack()).
void select_hot_pair(CsrDevice& A, CsrDevice& AT, int dev, cudaStream_t st);

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
int device_sm_count(int dev);

// Marks the two operands of an iteration L2-resident when their tile records
// and `vector_bytes` of per-iteration vectors fit in kL2ResidentShare of the
// device's L2: their bulk copies then load with an evict-last policy, so the
// next product reads them from L2 instead of HBM.  Larger operands keep the
// evict-first policy (streamed once per product).
constexpr double kL2ResidentShare = 0.85;
void mark_l2_resident(CsrDevice& A, CsrDevice& AT, double vector_bytes, int dev);

// Launch autotuner (results remembered per device, operand signature and
// timed product: shape, crossing and empty rows, hot slots, option, `kind`):
// times the product of `A` at 1-4 resident blocks per SM and, for an operand
// without hot slots, with L2 and with L1-cached gathers, and records the
// fastest median of three bursts in A.tuned_blocks_per_sm and A.gather_l1
// (operands with fewer than 4 tiles per SM keep the default grid and L2
// gathers).  `launch`, when given, launches the product that will run (its
// fused epilogue writing scratch copies of the iterates) for the candidate set
// in the view; `kind` names it in the remembered results.  Without it the
// store-only product is timed.  gather_cache is the option of that name: -1
// keeps L2 gathers, 1 takes L1-cached gathers without timing them, 0 times both.
using TuneLaunch = std::function<void(const CsrView&)>;
// launch_blocks > 0 fixes the blocks per SM (capped by what fits): only the
// gather modes are timed, and nothing when there is one candidate.
void autotune_operand(CsrDevice& A, cudaStream_t st, int dev, int* status, int gather_cache,
                      const TuneLaunch& launch = {}, int kind = 0, int launch_blocks = 0);

constexpr int kSpmvWarps = 4;     // warps per block (each with its own ring)
constexpr int kSpmvStages = 2;    // ring depth per warp
// Hot-slot kernel: one block per SM of kSpmvHotWarps warps (aliased staging,
// ~109 KB) plus the 48 KB FP32 hot copy, which keeps the 164 KB shared-memory
// carve-out and so ~92 KB of L1 for the outstanding cold gathers.  Measured on
// the 2,000,000 x 5,000,000 Zipf LP (A^T y per launch): 11 warps with a 16 K-slot
// copy 0.390 ms, 13 warps with 12 K slots 0.386 ms, 14 warps with 8 K slots
// 0.412 ms (earlier kernel generation: 8 warps / 16 K 0.548 ms, 11 / 16 K 0.459
// ms, no hot slots 0.505 ms).
constexpr int kSpmvHotWarps = 13;
constexpr int kSpmvHotCap = 12288;            // most hot slots (48 KB FP32 copy)
constexpr int kSpmvHotMinUses = 2;            // gathers per slot per resident block
constexpr double kSpmvHotMinShare = 0.15;     // share of the non-zeros the slots must take

// Launches `k` with programmatic stream serialization, so that it may start
// while the previous kernel of the stream finishes (the kernels wait with
// grid_dep_wait() before touching anything that kernel may write).
template <typename... KArgs, typename... Args>
void launch_dependent(void (*k)(KArgs...), int grid, int block, size_t smem, cudaStream_t st, Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(unsigned(grid));
    cfg.blockDim = dim3(unsigned(block));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    PB_CUDA_CHECK(cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...));
}

template <class Epi, typename AccT, typename XT, bool kLo>
struct SpmvLauncher {
    using L = SpmvSmemLayout<kSpmvWarps, kSpmvStages, kLo, AccT>;
    template <bool kRowMap>
    static constexpr auto kernel() {
        return &spmv_warp_kernel<Epi, AccT, XT, kLo, kRowMap, kSpmvWarps, kSpmvStages>;
    }
    template <bool kRowMap>
    static constexpr auto l1_kernel() {
        return &spmv_warp_kernel<Epi, AccT, XT, kLo, kRowMap, kSpmvWarps, kSpmvStages, kGatherL1>;
    }
    // Operands with hot slots: FP32 gathers use the shared-memory copy
    // (kGatherHot, kSpmvHotWarps warps per block); wider gathers resolve the
    // slots through hot_idx with the plain layout (kGatherHotIdx).
    static constexpr int kHotMode = sizeof(XT) == 4 ? kGatherHot : kGatherHotIdx;
    static constexpr int kHotWarps = kHotMode == kGatherHot ? kSpmvHotWarps : kSpmvWarps;
    using LH = SpmvSmemLayout<kHotWarps, kSpmvStages, kLo, AccT, kHotMode == kGatherHot>;
    static constexpr size_t kHotSmem =
        LH::bytes + (kHotMode == kGatherHot ? size_t(kSpmvHotCap) * sizeof(XT) : 0);
    template <bool kRowMap>
    static constexpr auto hot_kernel() {
        return &spmv_warp_kernel<Epi, AccT, XT, kLo, kRowMap, kHotWarps, kSpmvStages, kHotMode>;
    }
    // Resident blocks per SM the hot kernel is configured for.
    static constexpr int kHotTargetBlocks =
        kHotMode == kGatherHot
            ? (int((228 * 1024) / (kHotSmem + 1024)) > 0 ? int((228 * 1024) / (kHotSmem + 1024)) : 1)
                      : (int((132 * 1024) / (L::bytes + 1024)) > 0 ? int((132 * 1024) / (L::bytes + 1024)) : 1);
    // Default resident blocks per SM: as many as fit in ~132 KB of shared
    // memory, which leaves ~100 KB of L1 for outstanding gather misses.
    static constexpr int kTargetBlocks =
        int((132 * 1024) / (L::bytes + 1024)) > 0 ? int((132 * 1024) / (L::bytes + 1024)) : 1;

    // Dense variants: the finished rows are staged over the tile's own slots
    // (no per-warp row buffer), and the carve-out is sized for kDenseBlocks
    // blocks, so more warps hide the gather and epilogue latencies when the
    // gathers need less L1 (local operands).  Chosen by a tuned grid of more
    // than kTargetBlocks blocks per SM.
    using LD = SpmvSmemLayout<kSpmvWarps, kSpmvStages, kLo, AccT, true>;
    static constexpr int kDenseBlocks =
        int((200 * 1024) / (LD::bytes + 1024)) < 6 ? int((200 * 1024) / (LD::bytes + 1024)) : 6;
    template <bool kRowMap, bool kL1>
    static constexpr auto dense_kernel() {
        return &spmv_warp_kernel<Epi, AccT, XT, kLo, kRowMap, kSpmvWarps, kSpmvStages,
                                 kL1 ? kGatherL1 : kGatherL2, true>;
    }
    template <bool kRowMap, bool kL1>
    static int dense_blocks_per_sm_impl(int dev) {
        static std::atomic<int> cache[64];
        if (dev < 0 || dev >= 64) dev = 0;
        int v = cache[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
        const auto k = dense_kernel<kRowMap, kL1>();
        PB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(LD::bytes)));
        const long long need = (long long)kDenseBlocks * (LD::bytes + 1024);
        int pct = int((need * 100 + 228 * 1024 - 1) / (228 * 1024));
        pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
        PB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        int nb = 0;
        PB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kSpmvWarps * 32, LD::bytes));
        if (nb < 1) nb = 1;
        cache[dev].store(nb, std::memory_order_relaxed);
        return nb;
    }
    // Most blocks per SM the dense variants reach (0 when they add none).
    static int dense_blocks_per_sm(int dev) {
        dense_blocks_per_sm_impl<true, true>(dev);
        dense_blocks_per_sm_impl<true, false>(dev);
        dense_blocks_per_sm_impl<false, true>(dev);
        const int nb = dense_blocks_per_sm_impl<false, false>(dev);
        return nb > kTargetBlocks ? nb : 0;
    }

    // kL1: the L1-cached variant (same layout and carve-out as the plain one).
    template <bool kRowMap, bool kL1 = false>
    static int blocks_per_sm_impl(int dev) {
        static std::atomic<int> cache[64];
        if (dev < 0 || dev >= 64) dev = 0;
        int v = cache[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
        const auto k = kL1 ? l1_kernel<kRowMap>() : kernel<kRowMap>();
        PB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(L::bytes)));
        // Carve-out for kTargetBlocks blocks (percent of the 228 KB maximum).
        const long long need = (long long)kTargetBlocks * (L::bytes + 1024);
        int pct = int((need * 100 + 228 * 1024 - 1) / (228 * 1024));
        pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
        PB_CUDA_CHECK(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        int nb = 0;
        PB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k, kSpmvWarps * 32, L::bytes));
        if (nb < 1) nb = 1;
        cache[dev].store(nb, std::memory_order_relaxed);
        return nb;
    }
    template <bool kRowMap>
    static int hot_blocks_per_sm_impl(int dev) {
        static std::atomic<int> cache[64];
        if (dev < 0 || dev >= 64) dev = 0;
        int v = cache[dev].load(std::memory_order_relaxed);
        if (v > 0) return v;
        PB_CUDA_CHECK(cudaFuncSetAttribute(hot_kernel<kRowMap>(),
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, int(kHotSmem)));
        const long long need = (long long)kHotTargetBlocks * (kHotSmem + 1024);
        int pct = int((need * 100 + 228 * 1024 - 1) / (228 * 1024));
        pct = pct < 1 ? 1 : (pct > 100 ? 100 : pct);
        PB_CUDA_CHECK(cudaFuncSetAttribute(hot_kernel<kRowMap>(),
                                           cudaFuncAttributePreferredSharedMemoryCarveout, pct));
        int nb = 0;
        PB_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, hot_kernel<kRowMap>(),
                                                                    kHotWarps * 32, kHotSmem));
        if (nb < 1) nb = 1;
        cache[dev].store(nb, std::memory_order_relaxed);
        return nb;
    }
    // Queries occupancy (and sets the shared-memory attributes) for all
    // variants; call before any stream capture.
    static int blocks_per_sm(int dev) {
        dense_blocks_per_sm(dev);
        blocks_per_sm_impl<true>(dev);
        blocks_per_sm_impl<true, true>(dev);
        blocks_per_sm_impl<false, true>(dev);
        hot_blocks_per_sm_impl<true>(dev);
        hot_blocks_per_sm_impl<false>(dev);
        return blocks_per_sm_impl<false>(dev);
    }
    static int hot_blocks_per_sm(int dev) {
        hot_blocks_per_sm_impl<true>(dev);
        return hot_blocks_per_sm_impl<false>(dev);
    }
    // Grid for one launch: A.blocks_per_sm (autotuned) or the default target,
    // never more than fit, never more blocks than tile groups.
    // For an operand with hot slots the tuned value applies to the FP32 hot
    // kernel (the one the tuner times); the kGatherHotIdx kernels use the default.
    // True when the launch takes a dense variant.
    static bool dense_launch(const CsrView& A) { return A.hot == 0 && A.blocks_per_sm > kTargetBlocks; }
    static int grid_for(const CsrView& A, int dev) {
        const bool mapped = A.row_map != nullptr;
        const bool hot = A.hot > 0;
        int occ;
        if (hot) occ = mapped ? hot_blocks_per_sm_impl<true>(dev) : hot_blocks_per_sm_impl<false>(dev);
        else if (dense_launch(A))
            occ = mapped ? (A.gather_l1 ? dense_blocks_per_sm_impl<true, true>(dev) : dense_blocks_per_sm_impl<true, false>(dev))
                         : (A.gather_l1 ? dense_blocks_per_sm_impl<false, true>(dev) : dense_blocks_per_sm_impl<false, false>(dev));
        else occ = mapped ? blocks_per_sm_impl<true>(dev) : blocks_per_sm_impl<false>(dev);
        int bps;
        if (hot) bps = (kHotMode == kGatherHot && A.blocks_per_sm > 0) ? A.blocks_per_sm : kHotTargetBlocks;
        else bps = A.blocks_per_sm > 0 ? A.blocks_per_sm : kTargetBlocks;
        bps = bps < occ ? bps : occ;
        const int warps = hot ? kHotWarps : kSpmvWarps;
        const long long cap = (long long)bps * device_sm_count(dev);
        const long long need = (A.num_tiles + warps - 1) / warps;
        return int(need < cap ? need : cap);
    }
    static void launch(const CsrView& A, const XT* x, const Epi& epi, int* dev_status,
                       cudaStream_t st, int dev) {
        if (A.rows <= 0) return;
        if (A.num_tiles > 0) {
            const bool mapped = A.row_map != nullptr;
            const int grid = grid_for(A, dev);
            if (A.hot > 0) {
                if (A.hot > kSpmvHotCap || A.hot_idx == nullptr) throw std::logic_error("SpmvLauncher: bad hot slots");
                if (mapped)
                    launch_dependent(hot_kernel<true>(), grid, kHotWarps * 32, kHotSmem, st, A, x, epi, dev_status);
                else
                    launch_dependent(hot_kernel<false>(), grid, kHotWarps * 32, kHotSmem, st, A, x, epi, dev_status);
            } else if (dense_launch(A)) {
                const size_t sm = LD::bytes;
                if (mapped) {
                    if (A.gather_l1) launch_dependent(dense_kernel<true, true>(), grid, kSpmvWarps * 32, sm, st, A, x, epi, dev_status);
                    else launch_dependent(dense_kernel<true, false>(), grid, kSpmvWarps * 32, sm, st, A, x, epi, dev_status);
                } else {
                    if (A.gather_l1) launch_dependent(dense_kernel<false, true>(), grid, kSpmvWarps * 32, sm, st, A, x, epi, dev_status);
                    else launch_dependent(dense_kernel<false, false>(), grid, kSpmvWarps * 32, sm, st, A, x, epi, dev_status);
                }
            } else if (A.gather_l1) {
                if (mapped)
                    launch_dependent(l1_kernel<true>(), grid, kSpmvWarps * 32, L::bytes, st, A, x, epi, dev_status);
                else
                    launch_dependent(l1_kernel<false>(), grid, kSpmvWarps * 32, L::bytes, st, A, x, epi, dev_status);
            } else if (mapped) {
                launch_dependent(kernel<true>(), grid, kSpmvWarps * 32, L::bytes, st, A, x, epi, dev_status);
            } else {
                launch_dependent(kernel<false>(), grid, kSpmvWarps * 32, L::bytes, st, A, x, epi, dev_status);
            }
        }
        const int fix = A.num_cross + A.num_empty;
        if (fix > 0) {
            const int grid = (fix + 255) / 256 < 2048 ? (fix + 255) / 256 : 2048;
            launch_dependent(&spmv_fixup_kernel<Epi, AccT>, grid, 256, 0, st, A, epi);
        }
    }
    // Kernels one launch() call issues.
    static int launches(const CsrView& A) {
        if (A.rows <= 0) return 0;
        return (A.num_tiles > 0 ? 1 : 0) + (A.num_cross + A.num_empty > 0 ? 1 : 0);
    }
};

}  // namespace pb
