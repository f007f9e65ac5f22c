// noalloc.cu — y = A x over a caller-owned device CSR without allocating.
//
// Some callers cannot call cudaMalloc at the point where they need a sparse
// product: a branch-and-bound or rolling-horizon driver that has sized all of
// its device memory up front and runs under a fixed budget, code that runs
// while a stream is being captured into a CUDA graph (cudaMalloc is not a
// stream operation and cudaFree synchronises the device), and hosts that own
// the device memory pool and hand the library only pointers.  For them this
// file provides one entry point, pramaan_spmv_noalloc, that launches work on
// the caller's stream and allocates nothing: no cudaMalloc, no cudaFree, no
// allocating library routine.
//
// The product is the nnz-balanced ("merge-path") scheme of the library's main
// SpMV, restated for a plain CSR that has not been converted to the tiled
// format: each block takes T = 2048 consecutive entries, finds its rows by
// binary search in row_ptr, and combines partial sums with a segmented block
// scan.  A row that crosses tile boundaries leaves one partial per tile in a
// scratch array; a second kernel adds each crossing row's partials in tile
// order.  That scratch is the file-scope array below: every GPU that loads
// the library holds it (512 KiB) until the process exits, it limits one call
// to kNoAllocMaxTiles tiles (nnz <= 134,217,728), and every call shares it,
// so calls that overlap on the GPU (on different streams) race; calls on one
// stream are ordered.  Every slot a call reads is written earlier in the same
// call, so nothing needs clearing between calls.
#include <atomic>
#include <mutex>
#include <string>

#include "common.cuh"

namespace pb {
namespace {

constexpr int kNaBlock = 256;
constexpr int kNaIpt = 8;
constexpr int kNaTile = kNaBlock * kNaIpt;           // 2048 entries per tile
constexpr int kNoAllocMaxTiles = 65536;              // nnz <= 65536 * 2048
constexpr int kNaRpCap = kNaTile + 8;                // row_ptr slice capacity

// Cross-tile partials: slot 2t holds the piece of the row that continues into
// tile t from earlier tiles (its last or a middle piece), slot 2t+1 the first
// piece of the row that begins in tile t and continues past it.
__device__ __align__(256) float g_noalloc_carry[2 * kNoAllocMaxTiles];

// Per device ordinal: the array's device address and the SM count, looked up
// once with that device current.  The address belongs to the runtime's primary
// context of the device, the one every call of this entry point uses.
std::atomic<float*> g_carry_addr[64];
std::atomic<int> g_sm_count[64];
std::mutex g_setup_mutex;

// row_ptr read with the padding convention: row m+1 ends at the padded end.
__device__ __forceinline__ int rp_at(const int* __restrict__ row_ptr, int m, int nnz_pad, int r) {
    return r <= m ? __ldg(row_ptr + r) : nnz_pad;
}

// max r in [0, m] with row_ptr[r] <= q
__device__ int row_holding(const int* __restrict__ row_ptr, int m, long long q) {
    int lo = 0, hi = m;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(row_ptr + mid) <= q) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void __launch_bounds__(kNaBlock)
    noalloc_spmv_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                        const float* __restrict__ val, int m, int n, int nnz,
                        const float* __restrict__ x, float* __restrict__ y,
                        float* __restrict__ carry) {
    __shared__ int s_rp[kNaRpCap];
    __shared__ int s_lohi[2];
    __shared__ int s_wrow[kNaBlock / 32];
    __shared__ float s_wval[kNaBlock / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nt = (nnz + kNaTile - 1) / kNaTile;
    const int nnz_pad = nt * kNaTile;
    const unsigned last_col = static_cast<unsigned>(n - 1);
    for (int t = blockIdx.x; t < nt; t += gridDim.x) {
        const int tile_base = t * kNaTile, tile_end = tile_base + kNaTile;
        if (tid == 0) {
            s_lohi[0] = t == 0 ? 0 : row_holding(row_ptr, m, tile_base);
            s_lohi[1] = t == nt - 1 ? m : row_holding(row_ptr, m, tile_end);
        }
        __syncthreads();
        const int r_lo = s_lohi[0], r_hi = s_lohi[1];
        const int cnt = r_hi - r_lo + 2;
        const bool in_smem = cnt >= 1 && cnt <= kNaRpCap;
        if (in_smem)
            for (int j = tid; j < cnt; j += kNaBlock) s_rp[j] = rp_at(row_ptr, m, nnz_pad, r_lo + j);
        __syncthreads();
        // Rows outside the loaded slice (reachable only when row_ptr is not
        // nondecreasing) are read from global memory, never past s_rp.
        auto rp = [&](int r) {
            const int j = r - r_lo;
            return (in_smem && j >= 0 && j < cnt) ? s_rp[j] : rp_at(row_ptr, m, nnz_pad, r);
        };

        const int k0 = tile_base + tid * kNaIpt, k1 = k0 + kNaIpt;
        float p[kNaIpt];
#pragma unroll
        for (int j = 0; j < kNaIpt; ++j) {
            const int k = k0 + j;
            if (k < nnz) {
                unsigned c = static_cast<unsigned>(__ldg(col + k));
                c = c < last_col ? c : last_col;   // malformed input never reads out of bounds
                p[j] = __ldg(val + k) * __ldg(x + c);
            } else {
                p[j] = 0.0f;
            }
        }
        // first row whose end lies beyond k0 (thread 0 of tile 0 also owns rows ending at 0)
        int r;
        {
            int lo = r_lo, hi = r_hi;
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (rp(mid + 1) > k0) hi = mid; else lo = mid + 1;
            }
            r = (t == 0 && tid == 0) ? 0 : lo;
        }
        float acc = 0.0f, head_acc = 0.0f;
        int nemit = 0, head_row = -1;
        auto finish_row = [&](int row) {
            if (nemit == 0 && rp(row) < k0) { head_row = row; head_acc = acc; }
            else y[row] = acc;
            ++nemit;
            acc = 0.0f;
        };
#pragma unroll
        for (int j = 0; j < kNaIpt; ++j) {
            while (r < m && r <= r_hi && rp(r + 1) <= k0 + j) { finish_row(r); ++r; }
            acc += p[j];
        }
        while (r < m && r <= r_hi && rp(r + 1) <= k1) { finish_row(r); ++r; }

        // segmented block scan of (tail row, tail partial)
        int krow = r;
        float kval = acc;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int ro = __shfl_up_sync(0xffffffffu, krow, d);
            const float vo = __shfl_up_sync(0xffffffffu, kval, d);
            if (lane >= d && ro == krow) kval += vo;
        }
        if (lane == 31) { s_wrow[warp] = krow; s_wval[warp] = kval; }
        __syncthreads();
        int prow = -1;
        float pval = 0.0f;
        for (int w = 0; w < warp; ++w) {
            if (s_wrow[w] == prow) pval += s_wval[w]; else { prow = s_wrow[w]; pval = s_wval[w]; }
        }
        if (krow == prow) kval += pval;
        int erow = __shfl_up_sync(0xffffffffu, krow, 1);
        float eval = __shfl_up_sync(0xffffffffu, kval, 1);
        if (lane == 0) { erow = prow; eval = pval; }

        if (head_row >= 0) {
            const float tot = head_acc + (erow == head_row ? eval : 0.0f);
            if (rp(head_row) >= tile_base) y[head_row] = tot;
            else carry[2 * t] = tot;                 // last piece of a crossing row
        }
        if (tid == kNaBlock - 1 && krow < m && rp(krow) < tile_end && rp(krow + 1) > tile_end) {
            carry[2 * t + (rp(krow) >= tile_base ? 1 : 0)] = kval;   // first or middle piece
        }
        __syncthreads();
    }
}

// For every tile where a crossing row begins: add the row's pieces in tile order.
__global__ void noalloc_fixup_kernel(const int* __restrict__ row_ptr, int m, int nnz,
                                     const float* __restrict__ carry, float* __restrict__ y) {
    const int nt = (nnz + kNaTile - 1) / kNaTile;
    const int nnz_pad = nt * kNaTile;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt - 1; t += gridDim.x * blockDim.x) {
        const long long tile_base = t * (long long)kNaTile, tile_end = tile_base + kNaTile;
        const int R = row_holding(row_ptr, m, tile_end - 1);
        if (R >= m) continue;
        const int start = rp_at(row_ptr, m, nnz_pad, R), end = rp_at(row_ptr, m, nnz_pad, R + 1);
        if (start < tile_base || end <= tile_end) continue;
        const int t1 = (end - 1) / kNaTile;
        float sum = carry[2 * t + 1];
        for (int tt = t + 1; tt <= t1; ++tt) sum += carry[2 * tt];
        y[R] = sum;
    }
}

// Device address of the scratch array for `dev` (and its SM count), looked up
// once per device with that device current and cached.  With lazy module
// loading this first lookup is also where the module, and with it the array,
// may be loaded onto the device.
float* carry_address(int dev, int* sms) {
    if (dev < 0 || dev >= 64) throw InvalidArgument("device ordinal out of range");
    float* p = g_carry_addr[dev].load(std::memory_order_acquire);
    if (p) {
        *sms = g_sm_count[dev].load(std::memory_order_relaxed);
        return p;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_carry_addr[dev].load(std::memory_order_relaxed);
    if (!p) {
        int count = 0;
        PB_CUDA_CHECK(cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev));
        void* addr = nullptr;
        PB_CUDA_CHECK(cudaGetSymbolAddress(&addr, g_noalloc_carry));
        p = static_cast<float*>(addr);
        g_sm_count[dev].store(count, std::memory_order_relaxed);
        g_carry_addr[dev].store(p, std::memory_order_release);
    }
    *sms = g_sm_count[dev].load(std::memory_order_relaxed);
    return p;
}

}  // namespace

// Host side of pramaan_spmv_noalloc; errors become exceptions handled by the
// extern "C" wrapper in abi.cu.
void spmv_noalloc(const int32_t* d_row_ptr, const int32_t* d_col_idx, const float* d_values,
                  int32_t m, int32_t n, int32_t nnz, const float* d_x, float* d_y,
                  cudaStream_t stream) {
    if (m < 0 || n < 0 || nnz < 0) throw InvalidArgument("negative dimension");
    if (nnz > (long long)kNoAllocMaxTiles * kNaTile)
        throw InvalidArgument("pramaan_spmv_noalloc: nnz " + std::to_string(nnz) +
                              " exceeds the scratch limit of " +
                              std::to_string((long long)kNoAllocMaxTiles * kNaTile) + " entries");
    if (m == 0) return;
    if (!d_row_ptr || !d_y) throw InvalidArgument("row_ptr and y must not be NULL");
    if (nnz > 0 && (!d_col_idx || !d_values || !d_x || n == 0))
        throw InvalidArgument("col_idx, values and x must not be NULL (and n > 0) when nnz > 0");
    int dev = 0;
    PB_CUDA_CHECK(cudaGetDevice(&dev));
    int sms = 0;
    float* carry = carry_address(dev, &sms);
    if (nnz == 0) {
        PB_CUDA_CHECK(cudaMemsetAsync(d_y, 0, size_t(m) * sizeof(float), stream));
        return;
    }
    const int nt = (nnz + kNaTile - 1) / kNaTile;
    const int grid = nt < 8 * sms ? nt : 8 * sms;
    noalloc_spmv_kernel<<<grid, kNaBlock, 0, stream>>>(d_row_ptr, d_col_idx, d_values, m, n, nnz,
                                                       d_x, d_y, carry);
    PB_CUDA_CHECK(cudaGetLastError());
    if (nt > 1) {
        const int fgrid = (nt + 255) / 256;
        noalloc_fixup_kernel<<<fgrid, 256, 0, stream>>>(d_row_ptr, m, nnz, carry, d_y);
        PB_CUDA_CHECK(cudaGetLastError());
    }
}

}  // namespace pb
