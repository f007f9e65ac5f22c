// panel.cuh — column-panel product for the long rows of an operand whose
// row lengths follow a power law (the A x̄ product of the dual update).
//
// Why.  On a uniform-random column pattern every non-zero gathers one x̄
// entry from a random L2 sector, and B200 serves those at one sector request
// per SM per clock (gather_ceiling_kernel, ceiling.cu): the tiled product of
// a 108 M-entry Zipf LP is bound by that rate at about a third of HBM
// bandwidth.  The long rows of such an operand hold most of its non-zeros
// (rows of 296 or more entries hold ~76 % of a Zipf(1.5) LP's), and every one
// of them touches almost every part of x̄.  So x̄ is cut into P column panels,
// one per SM, each small enough for shared memory; block p loads panel p of
// x̄ once per product and streams the entries of all long rows that fall in
// its panel, gathering from shared memory instead of L2.  Each long row then
// has one partial sum per panel, written densely (part[p * L + r]); a finish
// kernel adds a row's P partials in panel order and applies the row's
// epilogue.  The short rows keep the tiled product (their own operand, which
// skips the long rows).
//
// Panel records (built once per operand, panel.cu)
//   Panel p's entries are the entries of the long rows with a column in
//   [p W, (p+1) W), ordered by long row and, within a row, in CSR order; the
//   entries of long row r in panel p form segment (p, r), possibly empty.  A
//   panel's segments are cut into chunks of at most kPanelEnt entries and
//   kPanelSegCap segments (a segment never straddles two chunks), each one
//   record of PanelRec::bytes (1,856 for 256 entries, 7.25 bytes per entry):
//     col   u16[256]   column minus p W (panel_col_slot; padding 0)
//     val   f32[256]   values (FP32), lane-interleaved 16-byte chunks
//                      (panel_val_slot; padding 0)
//     bits  u32[8]     bit q: entry q is the first entry of a segment (also
//                      set at the first padding entry, which so starts a run
//                      no segment reads)
//     seg   u16[129]   entry offset of each segment of the chunk, then nent
//     head  int4       {first segment (long-row index), segments, entries, 0}
//   chunk_ptr[p] .. chunk_ptr[p+1] are panel p's records.
//
// Sums.  Lane l owns entries 8 l .. 8 l + 7.  It forms the segmented prefix
// of its entries (restarting at every segment start and at its first entry)
// with FMAs in entry order and stores it in shared memory over the chunk's
// value slots (already in registers).  A segment [a, b) is then the sum of its
// pieces, one per lane it touches, each the prefix at the piece's last entry,
// added in entry order.  Every sum has a fixed order, so results are
// bit-identical from run to run.
//
// Shape.  One block of kPanelWarps warps per SM, each warp with a
// kPanelStages-deep ring of records filled by bulk copies and its next
// kPanelPrefetch records prefetched into L2; the panel of x takes the rest of
// the shared memory (W <= 35,744 columns).  Short per-lane chains and many
// warps: the kernel is bound by dependent-instruction latency before HBM
// (measured: 12 warps with 16 entries per lane issued 48 % of cycles, mostly
// waiting on fixed-latency dependencies).
#pragma once

#include "csr_device.cuh"

namespace pb {

constexpr int kPanelIpt = 8;                  // entries per lane
constexpr int kPanelEnt = 32 * kPanelIpt;     // entries per chunk record (256)
constexpr int kPanelSegCap = 128;             // segments per chunk record
constexpr int kPanelWarps = 24;               // warps per panel block (one block per SM)
constexpr int kPanelStages = 2;               // ring depth per warp
constexpr int kPanelPrefetch = 2;             // records each warp has prefetched into L2 beyond its ring

struct PanelRec {
    static constexpr size_t off_col = 0;                             // u16[256]
    static constexpr size_t off_val = 2 * kPanelEnt;                 // f32[256]
    static constexpr size_t off_bits = off_val + 4 * kPanelEnt;      // u32[8]
    static constexpr size_t off_seg = off_bits + kPanelEnt / 8;      // u16[129], padded to 16 bytes
    static constexpr size_t off_head = (off_seg + 2 * (kPanelSegCap + 1) + 15) / 16 * 16;   // int4
    static constexpr size_t bytes = off_head + 16;
    static_assert(bytes == 1856 && bytes % 16 == 0, "panel record layout");
};

// Slot of chunk-local entry q in the record's u16 column array: lane q / 8
// reads its 8 columns as one 16-byte chunk (unit q / 8), so a warp reads 512
// contiguous bytes.
__host__ __device__ constexpr int panel_col_slot(int q) { return q; }
// Slot of entry q in the value array (and of its prefix, see below): lane l
// reads its 8 values as two 16-byte chunks; chunk k of lane l is unit k * 32 + l.
__host__ __device__ constexpr int panel_val_slot(int q) {
    return (((q % kPanelIpt) / 4) * 32 + q / kPanelIpt) * 4 + (q % 4);
}
static_assert(panel_val_slot(0) == 0 && panel_val_slot(4) == 128 && panel_val_slot(8) == 4 &&
                  panel_val_slot(255) == 255,
              "panel_val_slot layout");

// Device view of one operand's panel split.
// The same kernel serves two layouts:
//   * the A x̄ split (vec_idx null): block p gathers from x̄[p W, p W + W),
//     its segments are the long rows, and segment s of panel p is written to
//     part[p * L + s];
//   * the hot part of Aᵀy (vec_idx set): every block gathers from the
//     vec_len entries x[vec_idx[k]] (y of the longest rows of A), its
//     segments are the W columns of its panel, and segment s of panel p is
//     written to part[p * W + s] (the column itself).
struct PanelView {
    int panels = 0;       // P (one block each)
    int width = 0;        // columns per panel W (a multiple of 4)
    int cols = 0;         // columns of the operand
    int long_rows = 0;    // L (A x̄ split) or 0
    const unsigned char* rec = nullptr;   // chunk records, panel-major
    const int* chunk_ptr = nullptr;       // [P + 1]
    const int* long_row = nullptr;        // [L] original row of every long row
    float* part = nullptr;                // [P * out_stride] per-panel sums
    int out_stride = 0;                   // L or W
    const int* vec_idx = nullptr;         // [vec_len] gathered vector entries (hot part of Aᵀy)
    int vec_len = 0;
};

// Shared memory of the panel kernel: the warps' rings, their mbarriers, then
// the block's panel of x (width floats).
struct PanelSmem {
    static constexpr size_t ring_bytes = size_t(kPanelWarps) * kPanelStages * PanelRec::bytes;
    static constexpr size_t off_bar = ring_bytes;
    static constexpr size_t off_x = (off_bar + size_t(kPanelWarps) * kPanelStages * 8 + 127) / 128 * 128;
    static constexpr size_t max_bytes = 232448;   // 227 KB: the opt-in maximum per block on sm_100
    static constexpr int max_width = int((max_bytes - off_x) / 4) / 4 * 4;
    static size_t bytes(int width) { return off_x + size_t(width) * 4; }
};

// Launches the panel kernel over view `v` (grid: one block per panel) as a
// dependent launch on `st`.
void panel_product_launch(const PanelView& v, const float* x, int* dev_status, cudaStream_t st);

// Adds the P partials of every long row in panel order and applies the row's
// epilogue (the same epilogue object as the short rows' tiled product).  One
// thread per row, 8 partials in flight at a time (measured on the 2 M x 5 M
// Zipf LP: 28 us per launch, against 39 us with 16 predicated loads in flight
// and 48 us with four threads per row).
template <class Epi>
__global__ void __launch_bounds__(256) panel_finish_kernel(const PanelView P, const Epi epi) {
    grid_dep_launch();
    grid_dep_wait();
    typename Epi::State est;
    epi.init(est);
    const int L = P.long_rows;
    const size_t ld = size_t(L);
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < L; r += gridDim.x * blockDim.x) {
        const float* pp = P.part + r;
        float sum = 0.f;
        int q = 0;
        for (; q + 8 <= P.panels; q += 8) {
            float v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) v[u] = __ldcg(pp + size_t(q + u) * ld);
#pragma unroll
            for (int u = 0; u < 8; ++u) sum += v[u];
        }
        for (; q < P.panels; ++q) sum += __ldcg(pp + size_t(q) * ld);
        epi.apply(est, P.long_row[r], sum);
    }
    epi.finish(est, 1);
}

// The panel split of one operand: the short rows as their own tiled operand,
// the long rows as panel records.
struct PanelSplit {
    bool active = false;
    int panels = 0, width = 0, long_rows = 0, min_len = 0, num_chunks = 0;
    long long long_nnz = 0;
    CsrDevice S;                        // short rows (long rows neither computed nor written)
    DevBuf<unsigned char> rec;
    DevBuf<int> chunk_ptr, long_row;
    DevBuf<float> part;
    PanelView view(int cols) const {
        PanelView v;
        v.panels = panels; v.width = width; v.cols = cols; v.long_rows = long_rows;
        v.rec = rec.get(); v.chunk_ptr = chunk_ptr.get(); v.long_row = long_row.get(); v.part = part.get();
        v.out_stride = long_rows;
        return v;
    }
};

// Default row length from which a row is long: kPanelLenPerPanel x panels.
// Every long row costs one segment per panel (its partial written, read back
// and added by the finish kernel); every short row's entries cost a random L2
// gather each in the tiled product.  Measured on the 2,000,000 x 5,000,000
// Zipf LP (148 panels), A x̄ per launch: long from 74 entries 0.360 ms, 110
// 0.330, 148 0.327, 200 0.320, 260 0.316, 330 0.315, 420 0.322, 550 0.338,
// 700 0.348.
constexpr double kPanelLenPerPanel = 2.0;
// Auto mode takes the split when the long rows hold at least this share of
// the non-zeros and the operand has at least kPanelMinNnz of them.
constexpr double kPanelMinShare = 0.5;
constexpr long long kPanelMinNnz = 4LL << 20;

// The hot part of Aᵀy.  The rows of A whose y entries every column gathers
// most are the longest rows; their y entries fit in one block's shared memory
// (up to PanelSmem::max_width of them).  Block p holds those entries of y and
// streams, for the columns of its panel (the same panels as the A x̄ split),
// the hot rows' entries in column order: segment s of panel p is column
// p W + s, and part[p W + s] receives its sum over the hot rows.  The other
// entries of Aᵀ form the remaining operand, whose tiled product adds part[j]
// to its own sum in the primal update (EpiPrimalRefAdd).
struct PanelHot {
    bool active = false;
    int panels = 0, width = 0, hot_rows = 0, min_len = 0, num_chunks = 0;
    long long hot_nnz = 0;
    CsrDevice rest;                     // Aᵀ without the hot rows' entries
    DevBuf<unsigned char> rec;
    DevBuf<int> chunk_ptr, hot_row;
    DevBuf<float> part;                 // [P W]: per column, the sum over the hot rows
    PanelView view(int cols) const {
        PanelView v;
        v.panels = panels; v.width = width; v.cols = cols;
        v.rec = rec.get(); v.chunk_ptr = chunk_ptr.get(); v.part = part.get();
        v.out_stride = width;
        v.vec_idx = hot_row.get();
        v.vec_len = hot_rows;
        return v;
    }
};
// Rows shorter than this never count as hot rows of Aᵀy.
constexpr int kPanelHotMinLen = 32;

// Builds the hot part of Aᵀy for an operand whose A x̄ is split (`dual`
// active), from the flat A and Aᵀ (before pack()).  Leaves ph inactive when
// no row qualifies or a column has more hot entries than a chunk holds.  The
// remaining operand gets hot gather slots as any operand does (none with
// gather_cache -1).  Synchronises `st`.
void build_panel_hot(const CsrDevice& A, const CsrDevice& AT, const PanelSplit& dual, PanelHot& ph, int gather_cache,
                     int dev, cudaStream_t st);

// Builds the split of A (flat arrays, before A.pack()).  mode 0: automatic
// (power-law operands only); 1: whenever feasible, long rows from the default
// length; >= 2: whenever feasible, long rows from `mode` entries.  Feasible:
// at least one long row, panels of at most PanelSmem::max_width columns, no
// segment longer than kPanelEnt entries, P x L < 2^31.  Leaves ps inactive
// otherwise.  Synchronises `st`.
void build_panel_split(const CsrDevice& A, PanelSplit& ps, int mode, int dev, cudaStream_t st);

// Sets the panel kernel's shared-memory limit (call before any stream capture).
void panel_prepare(int dev);

// One product over the split: the panel kernel, the short rows' tiled product
// and the finish kernel, as dependent launches on `st`.
template <class Epi>
void panel_launch(const PanelSplit& ps, int cols, const float* x, const Epi& epi, int* dev_status,
                  cudaStream_t st, int dev) {
    const PanelView v = ps.view(cols);
    panel_product_launch(v, x, dev_status, st);
    SpmvLauncher<Epi, float, float, false>::launch(ps.S.view(false), x, epi, dev_status, st, dev);
    const int grid = (v.long_rows + 255) / 256 < 2048 ? (v.long_rows + 255) / 256 : 2048;
    launch_dependent(&panel_finish_kernel<Epi>, grid, 256, 0, st, v, epi);
}
template <class Epi>
int panel_launches(const PanelSplit& ps) {
    return 2 + SpmvLauncher<Epi, float, float, false>::launches(ps.S.view(false));
}

}  // namespace pb
