// csr_device.cu — uploads, FP32 hi/lo split, tiled-format construction and
// the on-device stable transpose for CsrDevice.
#include "csr_device.cuh"
#include "epilogues.cuh"

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <unordered_map>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

namespace pb {

int device_sm_count(int dev) {
    static std::atomic<int> cache[64];
    if (dev < 0 || dev >= 64) dev = 0;
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    int sms = 0;
    PB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cache[dev].store(sms, std::memory_order_relaxed);
    return sms;
}

namespace {

constexpr int kThreads = 256;
inline int grid_1d(long long n, int cap = 65535 * 8) {
    long long g = (n + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    return int(g < cap ? g : cap);
}

#define PB_GRID_STRIDE(i, n)                                                            \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n);       \
         i += (long long)gridDim.x * blockDim.x)

// Structural validation (the invariants CSRMatrix::validate enforces,
// include/pramaan/sparse_matrix.hpp:153-174).  Flag bit 1: row_ptr not monotone /
// bad ends; bit 2: column index out of range.
__global__ void validate_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                                int rows, int cols, int nnz, int* __restrict__ flag) {
    PB_GRID_STRIDE(i, (long long)rows + nnz + 1) {
        if (i < rows) {
            if (row_ptr[i] > row_ptr[i + 1]) atomicOr(flag, 1);
        } else if (i == rows) {
            if (row_ptr[0] != 0 || row_ptr[rows] != nnz) atomicOr(flag, 1);
        } else {
            const int c = col[i - rows - 1];
            if (c < 0 || c >= cols) atomicOr(flag, 2);
        }
    }
}

// val64 -> (hi, lo): hi = RN(v), lo = RN(v - hi); *inexact = 1 when any lo != 0.
__global__ void split_f64_kernel(const double* __restrict__ v, int nnz, float* __restrict__ hi,
                                 float* __restrict__ lo, int* __restrict__ inexact) {
    PB_GRID_STRIDE(k, nnz) {
        const double d = v[k];
        const float h = __double2float_rn(d);
        const float l = __double2float_rn(d - static_cast<double>(h));
        hi[k] = h;
        lo[k] = l;
        if (l != 0.0f) *inexact = 1;
    }
}

__global__ void nonempty_kernel(const int* __restrict__ row_ptr, int rows, int* __restrict__ ne) {
    PB_GRID_STRIDE(r, rows) ne[r] = row_ptr[r + 1] > row_ptr[r] ? 1 : 0;
}

// Compacted row pointer (non-empty rows, then nnz and nnz_pad), row map and
// the empty-row list.
__global__ void compact_rows_kernel(const int* __restrict__ row_ptr, const int* __restrict__ ne,
                                    const int* __restrict__ idx, int rows, int* __restrict__ rp_c,
                                    int* __restrict__ row_map, int* __restrict__ empty_rows) {
    PB_GRID_STRIDE(r, rows) {
        const int c = idx[r];
        if (ne[r]) {
            rp_c[c] = row_ptr[r];
            if (row_map) row_map[c] = static_cast<int>(r);
        } else if (empty_rows) {
            empty_rows[r - c] = static_cast<int>(r);
        }
    }
}

__global__ void rp_tail_kernel(int* __restrict__ rp_c, int rows_c, int nnz, int nnz_pad) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        rp_c[rows_c] = nnz;
        rp_c[rows_c + 1] = nnz_pad;
    }
}

// Row-start bitmap: one bit per entry at the first entry of every non-empty
// row, and at nnz when padding follows (the virtual padding row).
__global__ void flags_kernel(const int* __restrict__ rp_c, int rows_c, int nnz, int nnz_pad,
                             uint32_t* __restrict__ flags) {
    PB_GRID_STRIDE(c, (long long)rows_c + 1) {
        int q;
        if (c < rows_c) q = rp_c[c];
        else if (nnz < nnz_pad) q = nnz;
        else continue;
        atomicOr(&flags[q >> 5], 1u << (q & 31));
    }
}

// Index of the compacted row holding entry q (rows_c + 2 pointer entries).
__device__ int row_of_entry(const int* __restrict__ rp_c, int rows_c, long long q) {
    int lo = 0, hi = rows_c;   // answer in [0, rows_c] (rows_c = virtual padding row)
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (rp_c[mid] <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// meta[t] = {first_row, tail_continues, 0, 0}
//   first_row      compacted row holding the tile's first entry
//   tail_continues 1 when the row holding the tile's last entry continues into
//                  the next tile
// begins[t] = 1 when that continuing row also begins in tile t: such a row is
// a crossing row, listed once, at the tile where it begins.
__global__ void meta_kernel(const int* __restrict__ rp_c, int rows_c, int tiles, int T,
                            int4* __restrict__ meta, int* __restrict__ begins) {
    PB_GRID_STRIDE(t, tiles) {
        const long long base = t * (long long)T, last = base + T - 1;
        const int fr = row_of_entry(rp_c, rows_c, base);
        const int tr = row_of_entry(rp_c, rows_c, last);
        const long long tend = rp_c[tr + 1];
        const int cont = (tr < rows_c && tend > last + 1) ? 1 : 0;
        meta[t] = make_int4(fr, cont, 0, 0);
        begins[t] = (cont && rp_c[tr] >= base) ? 1 : 0;
    }
}

// cross[idx[t]] = {original row, t, tiles touched} for every tile where a
// crossing row begins.
__global__ void cross_kernel(const int* __restrict__ rp_c, const int* __restrict__ row_map,
                             int rows_c, int tiles, int T, const int* __restrict__ begins,
                             const int* __restrict__ idx, int4* __restrict__ cross) {
    PB_GRID_STRIDE(t, tiles) {
        if (!begins[t]) continue;
        const long long last = t * (long long)T + T - 1;
        const int tr = row_of_entry(rp_c, rows_c, last);
        const long long tend = rp_c[tr + 1];
        const int span = int((tend - 1) / T - t + 1);
        cross[idx[t]] = make_int4(row_map ? row_map[tr] : tr, int(t), span, 0);
    }
}

// Writes the row index of every non-zero (one warp per row, coalesced).
__global__ void expand_rows_kernel(const int* __restrict__ row_ptr, int rows,
                                   int* __restrict__ row_of) {
    const int lane = threadIdx.x & 31;
    const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
    for (long long r = warp0; r < rows; r += nwarps) {
        const int b = row_ptr[r], e = row_ptr[r + 1];
        for (int k = b + lane; k < e; k += 32) row_of[k] = static_cast<int>(r);
    }
}

__global__ void iota_kernel(int* __restrict__ a, int n) {
    PB_GRID_STRIDE(k, n) a[k] = static_cast<int>(k);
}

// AT.row_ptr[c] = number of entries with sorted key < c (lower bound).
__global__ void keys_to_rowptr_kernel(const int* __restrict__ keys, int nnz, int cols,
                                      int* __restrict__ rp) {
    PB_GRID_STRIDE(c, (long long)cols + 1) {
        int lo = 0, hi = nnz;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (keys[mid] < c) lo = mid + 1; else hi = mid;
        }
        rp[c] = lo;
    }
}

// One block per tile: interleave the flat arrays into the tile record; an
// entry whose target has a hot slot stores ~slot.
__global__ void pack_kernel(const int* __restrict__ col, const float* __restrict__ val,
                            const uint32_t* __restrict__ flags, const int4* __restrict__ meta,
                            const int* __restrict__ slot, int tiles, unsigned char* __restrict__ rec) {
    constexpr int TW = TileRec::TW, FW = TileRec::FW;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
        unsigned char* r = rec + size_t(t) * TileRec::bytes;
        int* rc = reinterpret_cast<int*>(r + TileRec::off_col);
        float* rv = reinterpret_cast<float*>(r + TileRec::off_val);
        uint32_t* rf = reinterpret_cast<uint32_t*>(r + TileRec::off_flags);
        const size_t base = size_t(t) * TW;
        for (int k = threadIdx.x; k < TW; k += blockDim.x) {
            int c = col[base + k];
            if (slot) {
                const int h = slot[c];
                if (h >= 0) c = ~h;
            }
            rc[tile_slot(k)] = c;
            rv[tile_slot(k)] = val[base + k];
        }
        for (int k = threadIdx.x; k < FW; k += blockDim.x) rf[k] = flags[size_t(t) * FW + k];
        if (threadIdx.x == 0) *reinterpret_cast<int4*>(r + TileRec::off_meta) = meta[t];
    }
}

__global__ void permute_kernel(const int* __restrict__ perm, const int* __restrict__ row_of,
                               const float* __restrict__ val, const float* __restrict__ lo,
                               int nnz, int* __restrict__ t_col, float* __restrict__ t_val,
                               float* __restrict__ t_lo) {
    PB_GRID_STRIDE(k, nnz) {
        const int src = perm[k];
        t_col[k] = row_of[src];
        t_val[k] = val[src];
        if (t_lo) t_lo[k] = lo[src];
    }
}

// The FP32 remainders in the records' lane-interleaved order (tile_slot).
__global__ void interleave_lo_kernel(const float* __restrict__ src, long long n, float* __restrict__ dst) {
    PB_GRID_STRIDE(i, n) {
        const long long t = i / kSpmvTile;
        const int q = int(i - t * kSpmvTile);
        dst[t * kSpmvTile + tile_slot(q)] = src[i];
    }
}

__global__ void target_counts_kernel(const int* __restrict__ rp, int n, int* __restrict__ counts,
                                     int* __restrict__ ids) {
    PB_GRID_STRIDE(i, n) {
        counts[i] = rp[i + 1] - rp[i];
        ids[i] = int(i);
    }
}

__global__ void slot_scatter_kernel(const int* __restrict__ ids, int H, int* __restrict__ slot) {
    PB_GRID_STRIDE(k, H) slot[ids[k]] = int(k);
}

}  // namespace

namespace {

constexpr size_t kDeviceCacheCap = size_t(32) << 30;   // bytes kept per device
constexpr int kMaxDevices = 64;

struct DeviceCache {
    std::mutex mu;
    std::multimap<size_t, void*> free_blocks[kMaxDevices];   // by size
    size_t cached[kMaxDevices] = {};
    struct Block { size_t bytes; int dev; };
    std::unordered_map<void*, Block> live;                    // handed out
};

DeviceCache& device_cache() {
    static DeviceCache* c = new DeviceCache;   // kept to process exit
    return *c;
}

size_t cache_round(size_t b) {
    const size_t g = b < (size_t(1) << 20) ? 256 : (size_t(2) << 20);
    return (b + g - 1) / g * g;
}

}  // namespace

void* device_cache_alloc(size_t bytes) {
    int dev = 0;
    PB_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw std::runtime_error("device_cache_alloc: device ordinal out of range");
    const size_t want = cache_round(bytes);
    DeviceCache& c = device_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto& fb = c.free_blocks[dev];
        auto it = fb.lower_bound(want);
        if (it != fb.end() && it->first <= 2 * want) {
            void* p = it->second;
            const size_t sz = it->first;
            fb.erase(it);
            c.cached[dev] -= sz;
            c.live[p] = {sz, dev};
            return p;
        }
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaErrorMemoryAllocation) {
        (void)cudaGetLastError();
        device_cache_release(dev);
        e = cudaMalloc(&p, want);
    }
    PB_CUDA_CHECK(e);
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[p] = {want, dev};
    return p;
}

void device_cache_free(void* p) noexcept {
    DeviceCache& c = device_cache();
    DeviceCache::Block b{0, 0};
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.live.find(p);
        if (it == c.live.end()) return;
        b = it->second;
        c.live.erase(it);
    }
    int cur = -1;
    (void)cudaGetDevice(&cur);
    if (cur != b.dev) (void)cudaSetDevice(b.dev);
    // cudaFree waits for the device; a cached block must not be reused while
    // work issued before its release may still read or write it
    DeviceSyncScope gate;
    const cudaError_t e = cudaDeviceSynchronize();
    bool keep = e == cudaSuccess;
    if (keep) {
        std::lock_guard<std::mutex> lk(c.mu);
        if (c.cached[b.dev] + b.bytes <= kDeviceCacheCap) {
            c.free_blocks[b.dev].emplace(b.bytes, p);
            c.cached[b.dev] += b.bytes;
        } else {
            keep = false;
        }
    }
    if (!keep) (void)cudaFree(p);
    if (cur >= 0 && cur != b.dev) (void)cudaSetDevice(cur);
}

void device_cache_release(int dev) {
    DeviceCache& c = device_cache();
    std::vector<std::pair<int, void*>> out;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        for (int d = 0; d < kMaxDevices; ++d) {
            if (dev >= 0 && d != dev) continue;
            for (auto& kv : c.free_blocks[d]) out.emplace_back(d, kv.second);
            c.free_blocks[d].clear();
            c.cached[d] = 0;
        }
    }
    int cur = -1;
    (void)cudaGetDevice(&cur);
    DeviceSyncScope gate;
    for (auto& [d, p] : out) {
        if (d != cur) (void)cudaSetDevice(d);
        (void)cudaFree(p);
        if (d != cur && cur >= 0) (void)cudaSetDevice(cur);
    }
}

void CsrDevice::select_hot(const int* target_rp, int num_targets, int dev, cudaStream_t st) {
    hot = 0;
    hot_idx.reset();
    hot_slot.reset();
    if (packed || num_tiles == 0 || num_targets <= 0 || target_rp == nullptr) return;
    using Launch = SpmvLauncher<EpiStore<float, float>, float, float, false>;
    const int sms = device_sm_count(dev);
    // Each block of the hot kernel copies every slot once, so an operand with
    // few tiles per block gains nothing.
    const long long blocks = (long long)sms * Launch::kHotTargetBlocks;
    if ((long long)num_tiles < 64 * blocks * kSpmvHotWarps / 8) return;
    const int n = num_targets;
    DevBuf<int> counts{size_t(n)}, ids{size_t(n)}, counts_s{size_t(n)}, ids_s{size_t(n)};
    target_counts_kernel<<<grid_1d(n), kThreads, 0, st>>>(target_rp, n, counts.get(), ids.get());
    PB_CUDA_CHECK(cudaGetLastError());
    size_t tb = 0;
    PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, counts.get(), counts_s.get(), ids.get(),
                                                            ids_s.get(), n, 0, 32, st));
    DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
    PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairsDescending(temp.get(), tb, counts.get(), counts_s.get(), ids.get(),
                                                            ids_s.get(), n, 0, 32, st));
    const int H0 = n < kSpmvHotCap ? n : kSpmvHotCap;
    std::vector<int> hc(static_cast<size_t>(H0));
    PB_CUDA_CHECK(cudaMemcpyAsync(hc.data(), counts_s.get(), size_t(H0) * 4, cudaMemcpyDeviceToHost, st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
    const long long min_uses = (long long)kSpmvHotMinUses * blocks;
    long long covered = 0;
    int H = 0;
    while (H < H0 && (long long)hc[size_t(H)] >= min_uses) covered += hc[size_t(H++)];
    if (H == 0 || double(covered) < kSpmvHotMinShare * double(nnz)) return;
    hot_idx.alloc(size_t(H));
    PB_CUDA_CHECK(cudaMemcpyAsync(hot_idx.get(), ids_s.get(), size_t(H) * 4, cudaMemcpyDeviceToDevice, st));
    hot_slot.alloc(size_t(n));
    PB_CUDA_CHECK(cudaMemsetAsync(hot_slot.get(), 0xff, hot_slot.bytes(), st));   // -1: no slot
    slot_scatter_kernel<<<grid_1d(H), kThreads, 0, st>>>(ids_s.get(), H, hot_slot.get());
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaStreamSynchronize(st));   // temporaries are freed on return
    hot = H;
}

void select_hot_pair(CsrDevice& A, CsrDevice& AT, int dev, cudaStream_t st) {
    AT.select_hot(A.row_ptr.get(), A.rows, dev, st);
    A.select_hot(AT.row_ptr.get(), AT.rows, dev, st);
}

void CsrDevice::pack(cudaStream_t st) {
    if (packed) return;
    if (num_tiles > 0) {
        rec.alloc(size_t(num_tiles) * TileRec::bytes);
        const int grid = num_tiles < 65535 * 4 ? num_tiles : 65535 * 4;
        pack_kernel<<<grid, 256, 0, st>>>(col.get(), val.get(), flags.get(), meta.get(),
                                          hot > 0 ? hot_slot.get() : nullptr, num_tiles, rec.get());
        PB_CUDA_CHECK(cudaGetLastError());
        if (has_lo && val_lo.get()) {
            DevBuf<float> lo_i{size_t(nnz_pad)};
            interleave_lo_kernel<<<grid_1d(nnz_pad), kThreads, 0, st>>>(val_lo.get(), (long long)nnz_pad,
                                                                        lo_i.get());
            PB_CUDA_CHECK(cudaGetLastError());
            PB_CUDA_CHECK(cudaStreamSynchronize(st));
            val_lo = std::move(lo_i);
        }
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
    }
    hot_slot.reset();
    if (!keep_flat) {
        col.reset();
        val.reset();
    }
    flags.reset();
    meta.reset();
    packed = true;
}

void CsrDevice::allocate(int rows_, int cols_, int nnz_, bool lo) {
    if (rows_ < 0 || cols_ < 0 || nnz_ < 0) throw InvalidArgument("negative CSR dimension");
    rows = rows_; cols = cols_; nnz = nnz_;
    hot = 0;
    hot_idx.reset();
    hot_slot.reset();
    num_tiles = nnz > 0 ? ceil_div(nnz, kSpmvTile) : 0;
    nnz_pad = num_tiles * kSpmvTile;
    has_lo = lo;
    packed = false;
    rec.reset();
    row_ptr.alloc(size_t(rows) + 1);
    col.alloc(size_t(nnz_pad));
    val.alloc(size_t(nnz_pad));
    if (lo) val_lo.alloc(size_t(nnz_pad)); else val_lo.reset();
}

void CsrDevice::finalize(cudaStream_t st) {
    if (nnz_pad > nnz) {
        PB_CUDA_CHECK(cudaMemsetAsync(col.get() + nnz, 0, size_t(nnz_pad - nnz) * 4, st));
        PB_CUDA_CHECK(cudaMemsetAsync(val.get() + nnz, 0, size_t(nnz_pad - nnz) * 4, st));
        if (val_lo.get())
            PB_CUDA_CHECK(cudaMemsetAsync(val_lo.get() + nnz, 0, size_t(nnz_pad - nnz) * 4, st));
    }
    // ---- compact the non-empty rows ----
    DevBuf<int> ne(size_t(rows > 0 ? rows : 1)), idx(size_t(rows) + 1);
    rows_c = 0;
    if (rows > 0) {
        nonempty_kernel<<<grid_1d(rows), kThreads, 0, st>>>(row_ptr.get(), rows, ne.get());
        PB_CUDA_CHECK(cudaGetLastError());
        size_t tb = 0;
        PB_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, ne.get(), idx.get(), rows, st));
        DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
        PB_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(temp.get(), tb, ne.get(), idx.get(), rows, st));
        int last_idx = 0, last_ne = 0;
        PB_CUDA_CHECK(cudaMemcpyAsync(&last_idx, idx.get() + rows - 1, 4, cudaMemcpyDeviceToHost, st));
        PB_CUDA_CHECK(cudaMemcpyAsync(&last_ne, ne.get() + rows - 1, 4, cudaMemcpyDeviceToHost, st));
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
        rows_c = last_idx + last_ne;
    }
    num_empty = rows - rows_c;
    if (num_empty > 0) {
        row_map.alloc(size_t(rows_c > 0 ? rows_c : 1));
        empty_rows.alloc(size_t(num_empty));
    } else {
        row_map.reset();
        empty_rows.reset();
    }
    DevBuf<int> rp_c(size_t(rows_c) + 2);
    if (rows > 0) {
        compact_rows_kernel<<<grid_1d(rows), kThreads, 0, st>>>(
            row_ptr.get(), ne.get(), idx.get(), rows, rp_c.get(), num_empty > 0 ? row_map.get() : nullptr,
            num_empty > 0 ? empty_rows.get() : nullptr);
        PB_CUDA_CHECK(cudaGetLastError());
    }
    rp_tail_kernel<<<1, 1, 0, st>>>(rp_c.get(), rows_c, nnz, nnz_pad);
    PB_CUDA_CHECK(cudaGetLastError());

    // ---- row-start bitmap, tile descriptors, crossing rows ----
    flags.alloc(size_t(nnz_pad / 32 > 0 ? nnz_pad / 32 : 1));
    meta.alloc(size_t(num_tiles > 0 ? num_tiles : 1));
    PB_CUDA_CHECK(cudaMemsetAsync(flags.get(), 0, flags.bytes(), st));
    num_cross = 0;
    cross.reset();
    if (num_tiles > 0) {
        flags_kernel<<<grid_1d((long long)rows_c + 1), kThreads, 0, st>>>(rp_c.get(), rows_c, nnz,
                                                                         nnz_pad, flags.get());
        DevBuf<int> begins(static_cast<size_t>(num_tiles)), bidx(static_cast<size_t>(num_tiles));
        meta_kernel<<<grid_1d(num_tiles), kThreads, 0, st>>>(rp_c.get(), rows_c, num_tiles, kSpmvTile,
                                                             meta.get(), begins.get());
        PB_CUDA_CHECK(cudaGetLastError());
        size_t tb = 0;
        PB_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(nullptr, tb, begins.get(), bidx.get(), num_tiles, st));
        DevBuf<unsigned char> temp(tb > 0 ? tb : 1);
        PB_CUDA_CHECK(cub::DeviceScan::ExclusiveSum(temp.get(), tb, begins.get(), bidx.get(), num_tiles, st));
        int last_idx = 0, last_b = 0;
        PB_CUDA_CHECK(cudaMemcpyAsync(&last_idx, bidx.get() + num_tiles - 1, 4, cudaMemcpyDeviceToHost, st));
        PB_CUDA_CHECK(cudaMemcpyAsync(&last_b, begins.get() + num_tiles - 1, 4, cudaMemcpyDeviceToHost, st));
        PB_CUDA_CHECK(cudaStreamSynchronize(st));
        num_cross = last_idx + last_b;
        if (num_cross > 0) {
            cross.alloc(static_cast<size_t>(num_cross));
            cross_kernel<<<grid_1d(num_tiles), kThreads, 0, st>>>(
                rp_c.get(), num_empty > 0 ? row_map.get() : nullptr, rows_c, num_tiles, kSpmvTile,
                begins.get(), bidx.get(), cross.get());
            PB_CUDA_CHECK(cudaGetLastError());
        }
    }
    carry.alloc(size_t(2) * (num_tiles > 0 ? num_tiles : 1));
    PB_CUDA_CHECK(cudaMemsetAsync(carry.get(), 0, carry.bytes(), st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));   // temporaries are freed on return
}

static void upload_structure(CsrDevice& A, int rows, int cols, int nnz, const int* h_row_ptr,
                             const int* h_col, cudaStream_t st, int* d_flag) {
    PB_CUDA_CHECK(cudaMemcpyAsync(A.row_ptr.get(), h_row_ptr, (size_t(rows) + 1) * 4,
                                  cudaMemcpyHostToDevice, st));
    if (nnz > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(A.col.get(), h_col, size_t(nnz) * 4, cudaMemcpyHostToDevice,
                                      st));
    if (d_flag) {
        validate_kernel<<<grid_1d((long long)rows + nnz + 1), kThreads, 0, st>>>(
            A.row_ptr.get(), A.col.get(), rows, cols, nnz, d_flag);
        PB_CUDA_CHECK(cudaGetLastError());
    }
}

// Reads the validation flag; throws before any structure-dependent kernel runs.
static void check_structure(int* d_flag, cudaStream_t st) {
    if (!d_flag) return;
    int h = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&h, d_flag, 4, cudaMemcpyDeviceToHost, st));
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
    if (h & 1) throw InvalidArgument("row_ptr must start at 0, be non-decreasing and end at nnz");
    if (h & 2) throw InvalidArgument("col_idx entry out of bounds");
}

void csr_upload_f64(CsrDevice& A, int rows, int cols, int nnz, const int* h_row_ptr,
                    const int* h_col, const double* h_val, cudaStream_t st, int* d_flag) {
    A.allocate(rows, cols, nnz, /*lo=*/true);
    upload_structure(A, rows, cols, nnz, h_row_ptr, h_col, st, d_flag);
    check_structure(d_flag, st);
    if (nnz > 0) {
        DevBuf<double> v64{size_t(nnz)};
        DevBuf<int> inexact(1);
        PB_CUDA_CHECK(cudaMemsetAsync(inexact.get(), 0, 4, st));
        PB_CUDA_CHECK(cudaMemcpyAsync(v64.get(), h_val, size_t(nnz) * 8, cudaMemcpyHostToDevice, st));
        split_f64_kernel<<<grid_1d(nnz), kThreads, 0, st>>>(v64.get(), nnz, A.val.get(),
                                                            A.val_lo.get(), inexact.get());
        PB_CUDA_CHECK(cudaGetLastError());
        int h_inexact = 0;
        PB_CUDA_CHECK(cudaMemcpyAsync(&h_inexact, inexact.get(), 4, cudaMemcpyDeviceToHost, st));
        PB_CUDA_CHECK(cudaStreamSynchronize(st));   // v64 freed below
        if (!h_inexact) { A.val_lo.reset(); A.has_lo = false; }
    } else {
        A.val_lo.reset();
        A.has_lo = false;
    }
    A.finalize(st);
}

void csr_upload_f32(CsrDevice& A, int rows, int cols, int nnz, const int* h_row_ptr,
                    const int* h_col, const float* h_val, cudaStream_t st, int* d_flag) {
    A.allocate(rows, cols, nnz, /*lo=*/false);
    upload_structure(A, rows, cols, nnz, h_row_ptr, h_col, st, d_flag);
    check_structure(d_flag, st);
    if (nnz > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(A.val.get(), h_val, size_t(nnz) * 4, cudaMemcpyHostToDevice, st));
    A.finalize(st);
}

void mark_l2_resident(CsrDevice& A, CsrDevice& AT, double vector_bytes, int dev) {
    int l2 = 0;
    PB_CUDA_CHECK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    const double need = double(A.rec.bytes()) + double(AT.rec.bytes()) + vector_bytes;
    const int keep = (l2 > 0 && need <= kL2ResidentShare * double(l2)) ? 1 : 0;
    A.l2_resident = keep;
    AT.l2_resident = keep;
}

void csr_transpose(const CsrDevice& A, CsrDevice& AT, cudaStream_t st) {
    const int nnz = A.nnz;
    AT.allocate(A.cols, A.rows, nnz, A.has_lo);
    if (nnz == 0) {
        PB_CUDA_CHECK(cudaMemsetAsync(AT.row_ptr.get(), 0, (size_t(A.cols) + 1) * 4, st));
        AT.finalize(st);
        return;
    }
    DevBuf<int> row_of{size_t(nnz)}, keys_out{size_t(nnz)}, perm_in{size_t(nnz)}, perm_out{size_t(nnz)};
    expand_rows_kernel<<<grid_1d((long long)A.rows * 32), kThreads, 0, st>>>(A.row_ptr.get(), A.rows,
                                                                            row_of.get());
    PB_CUDA_CHECK(cudaGetLastError());
    iota_kernel<<<grid_1d(nnz), kThreads, 0, st>>>(perm_in.get(), nnz);
    PB_CUDA_CHECK(cudaGetLastError());
    int end_bit = 1;
    while (end_bit < 31 && (1LL << end_bit) < (long long)A.cols) ++end_bit;
    size_t temp_bytes = 0;
    PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, A.col.get(), keys_out.get(),
                                                  perm_in.get(), perm_out.get(), nnz, 0, end_bit, st));
    DevBuf<unsigned char> temp(temp_bytes > 0 ? temp_bytes : 1);
    PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(temp.get(), temp_bytes, A.col.get(), keys_out.get(),
                                                  perm_in.get(), perm_out.get(), nnz, 0, end_bit, st));
    keys_to_rowptr_kernel<<<grid_1d((long long)A.cols + 1), kThreads, 0, st>>>(keys_out.get(), nnz,
                                                                              A.cols, AT.row_ptr.get());
    PB_CUDA_CHECK(cudaGetLastError());
    permute_kernel<<<grid_1d(nnz), kThreads, 0, st>>>(
        perm_out.get(), row_of.get(), A.val.get(), A.has_lo ? A.val_lo.get() : nullptr, nnz,
        AT.col.get(), AT.val.get(), AT.has_lo ? AT.val_lo.get() : nullptr);
    PB_CUDA_CHECK(cudaGetLastError());
    AT.finalize(st);   // synchronises; temporaries are freed on return
}

// Launch autotuner: picks the resident blocks per SM and the gather mode for
// one operand by timing, for every candidate, the product that will run: the
// caller's fused launch on scratch copies of the vectors it writes, or, when
// none is given, the store-only product into scratch.  The candidates are
// timed round-robin, kTuneRepeats times each, and each keeps the median of its
// repeats, so one noisy burst cannot pick the shape.
namespace {

// Tuned launch shapes by operand signature and timed product, so repeated
// solves of the same operand (the same LP, or LPs of one generator and size)
// skip the timing.
struct TuneKey {
    int dev, rows, cols, nnz, tiles, cross, empty, hot, gather_cache, kind;
    bool operator<(const TuneKey& o) const {
        return std::tie(dev, rows, cols, nnz, tiles, cross, empty, hot, gather_cache, kind) <
               std::tie(o.dev, o.rows, o.cols, o.nnz, o.tiles, o.cross, o.empty, o.hot, o.gather_cache,
                        o.kind);
    }
};
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tuned;   // -> {blocks per SM, gather_l1}

constexpr int kTuneRepeats = 3;         // timed bursts per candidate
constexpr int kTuneBurst = 5;           // launches per burst
constexpr float kTuneMargin = 0.98f;    // a later candidate must be 2 % faster

}  // namespace

void autotune_operand(CsrDevice& A, cudaStream_t st, int dev, int* status, int gather_cache,
                      const TuneLaunch& launch, int kind, int launch_blocks) {
    using Epi = EpiStore<float, float>;
    using Launch = SpmvLauncher<Epi, float, float, false>;
    A.gather_l1 = (gather_cache > 0 && A.hot == 0) ? 1 : 0;
    if (A.num_tiles < 4 * device_sm_count(dev)) return;   // small operands: default grid
    if (!launch) kind = 0;
    const TuneKey key{dev, A.rows, A.cols, A.nnz, A.num_tiles, A.num_cross, A.num_empty, A.hot, gather_cache,
                      kind * 64 + (launch_blocks > 0 ? launch_blocks : 0)};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        const auto it = g_tuned.find(key);
        if (it != g_tuned.end()) {
            A.tuned_blocks_per_sm = it->second.first;
            A.gather_l1 = it->second.second;
            return;
        }
    }
    const int occ = A.hot > 0 ? Launch::hot_blocks_per_sm(dev) : Launch::blocks_per_sm(dev);
    // L1-cached gathers are a candidate for operands without hot slots; the
    // L2 mode comes first and is kept unless the other is 2 % faster.
    const int mode_lo = A.gather_l1;
    const int mode_hi = (gather_cache == 0 && A.hot == 0) ? 1 : A.gather_l1;
    DevBuf<float> xs, ys;
    if (!launch) {
        xs.alloc(static_cast<size_t>(A.cols > 0 ? A.cols : 1));
        ys.alloc(static_cast<size_t>(A.rows));
        PB_CUDA_CHECK(cudaMemsetAsync(xs.get(), 0, xs.bytes(), st));
    }
    const Epi epi{ys.get()};
    auto run = [&](const CsrView& v) {
        if (launch) launch(v);
        else Launch::launch(v, xs.get(), epi, status, st, dev);
    };
    // Grids above Launch::kTargetBlocks blocks per SM take the dense variants
    // (operands without hot slots).
    const int dense = A.hot > 0 ? 0 : Launch::dense_blocks_per_sm(dev);
    std::vector<std::pair<int, int>> cand;   // {gather mode, blocks per SM}
    for (int mode = mode_lo; mode <= mode_hi; ++mode) {
        if (launch_blocks > 0) {   // a fixed shape: the largest grid up to the request that fits
            const int top = std::max(std::min(occ, Launch::kTargetBlocks), dense);
            cand.push_back({mode, std::min(launch_blocks, top)});
            continue;
        }
        for (int bps = 1; bps <= occ && bps <= Launch::kTargetBlocks; ++bps) cand.push_back({mode, bps});
        for (int bps = Launch::kTargetBlocks + 1; bps <= dense; ++bps) cand.push_back({mode, bps});
    }
    if (cand.size() == 1) {   // nothing to time
        A.gather_l1 = cand[0].first;
        A.tuned_blocks_per_sm = cand[0].second;
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tuned[key] = {cand[0].second, cand[0].first};
        return;
    }
    std::vector<cudaEvent_t> ev(2 * cand.size() * kTuneRepeats);
    for (auto& e : ev) PB_CUDA_CHECK(cudaEventCreate(&e));
    for (const auto& c : cand) {   // warm-up of every shape
        A.gather_l1 = c.first;
        A.tuned_blocks_per_sm = c.second;
        run(A.view(false));
    }
    for (int r = 0; r < kTuneRepeats; ++r) {
        for (size_t k = 0; k < cand.size(); ++k) {
            A.gather_l1 = cand[k].first;
            A.tuned_blocks_per_sm = cand[k].second;
            const CsrView v = A.view(false);
            cudaEvent_t* e = &ev[2 * (k * kTuneRepeats + r)];
            PB_CUDA_CHECK(cudaEventRecord(e[0], st));
            for (int b = 0; b < kTuneBurst; ++b) run(v);
            PB_CUDA_CHECK(cudaEventRecord(e[1], st));
        }
    }
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
    float best = 1e30f;
    int best_bps = 0, best_mode = mode_lo;
    for (size_t k = 0; k < cand.size(); ++k) {
        float t[kTuneRepeats];
        for (int r = 0; r < kTuneRepeats; ++r) {
            cudaEvent_t* e = &ev[2 * (k * kTuneRepeats + r)];
            PB_CUDA_CHECK(cudaEventElapsedTime(&t[r], e[0], e[1]));
        }
        std::sort(t, t + kTuneRepeats);
        const float med = t[kTuneRepeats / 2];
        if (med < best * kTuneMargin) { best = med; best_bps = cand[k].second; best_mode = cand[k].first; }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    A.tuned_blocks_per_sm = best_bps;
    A.gather_l1 = best_mode;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = {best_bps, best_mode};
}

}  // namespace pb
