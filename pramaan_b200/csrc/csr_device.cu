// csr_device.cu — uploads, FP32 hi/lo split, tile schedule and the on-device
// stable transpose for CsrDevice.
#include "csr_device.cuh"

#include <cub/device/device_radix_sort.cuh>

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

// tile_row[t] = max r in [0, rows] with row_ptr[r] <= t*T (t in 1..tiles-1),
// tile_row[0] = 0, tile_row[tiles] = rows.
__global__ void tile_row_kernel(const int* __restrict__ row_ptr, int rows, int tiles, int T,
                                int* __restrict__ tile_row) {
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t <= tiles; t += gridDim.x * blockDim.x) {
        if (t == 0) { tile_row[0] = 0; continue; }
        if (t == tiles) { tile_row[t] = rows; continue; }
        const long long key = (long long)t * T;
        int lo = 0, hi = rows;   // answer in [0, rows]; row_ptr[0] = 0 <= key
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (row_ptr[mid] <= key) lo = mid; else hi = mid - 1;
        }
        tile_row[t] = lo;
    }
}

__global__ void fill_pad_kernel(int* __restrict__ row_ptr, int rows, int nnz_pad) {
    if (blockIdx.x == 0 && threadIdx.x == 0) row_ptr[rows + 1] = nnz_pad;
}

// Structural validation (the invariants CSRMatrix::validate enforces,
// include/pramaan/sparse_matrix.hpp:153-174).  Flag bit 1: row_ptr not monotone /
// bad end; bit 2: column index out of range.
__global__ void validate_kernel(const int* __restrict__ row_ptr, const int* __restrict__ col,
                                int rows, int cols, int nnz, int* __restrict__ flag) {
    const long long total = (long long)rows + nnz + 1;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
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

// val64 -> (hi, lo) with hi = RN(v), lo = RN(v - hi); flag bit 4 when any lo != 0.
__global__ void split_f64_kernel(const double* __restrict__ v, int nnz, float* __restrict__ hi,
                                 float* __restrict__ lo, int* __restrict__ inexact) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const double d = v[k];
        const float h = __double2float_rn(d);
        const float l = __double2float_rn(d - static_cast<double>(h));
        hi[k] = h;
        lo[k] = l;
        if (l != 0.0f) *inexact = 1;
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
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        a[k] = static_cast<int>(k);
}

// AT.row_ptr[c] = number of entries with sorted key < c (lower bound).
__global__ void keys_to_rowptr_kernel(const int* __restrict__ keys, int nnz, int cols,
                                      int* __restrict__ rp) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c <= cols;
         c += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = nnz;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (keys[mid] < c) lo = mid + 1; else hi = mid;
        }
        rp[c] = lo;
    }
}

__global__ void permute_kernel(const int* __restrict__ perm, const int* __restrict__ row_of,
                               const float* __restrict__ val, const float* __restrict__ lo,
                               int nnz, int* __restrict__ t_col, float* __restrict__ t_val,
                               float* __restrict__ t_lo) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < nnz;
         k += (long long)gridDim.x * blockDim.x) {
        const int src = perm[k];
        t_col[k] = row_of[src];
        t_val[k] = val[src];
        if (t_lo) t_lo[k] = lo[src];
    }
}

}  // namespace

void CsrDevice::allocate(int rows_, int cols_, int nnz_, bool lo) {
    if (rows_ < 0 || cols_ < 0 || nnz_ < 0) throw InvalidArgument("negative CSR dimension");
    rows = rows_; cols = cols_; nnz = nnz_;
    num_tiles = nnz > 0 ? ceil_div(nnz, kSpmvTile) : 0;
    nnz_pad = num_tiles * kSpmvTile;
    has_lo = lo;
    row_ptr.alloc(size_t(rows) + 2);
    col.alloc(size_t(nnz_pad));
    val.alloc(size_t(nnz_pad));
    if (lo) val_lo.alloc(size_t(nnz_pad)); else val_lo.reset();
    tile_row.alloc(size_t(num_tiles) + 1);
    counter.alloc(size_t(num_tiles > 0 ? num_tiles : 1));
    carry.alloc(size_t(2) * (num_tiles > 0 ? num_tiles : 1));
}

void CsrDevice::finalize(cudaStream_t st) {
    fill_pad_kernel<<<1, 1, 0, st>>>(row_ptr.get(), rows, nnz_pad);
    PB_CUDA_CHECK(cudaGetLastError());
    if (nnz_pad > nnz) {
        PB_CUDA_CHECK(cudaMemsetAsync(col.get() + nnz, 0, size_t(nnz_pad - nnz) * 4, st));
        PB_CUDA_CHECK(cudaMemsetAsync(val.get() + nnz, 0, size_t(nnz_pad - nnz) * 4, st));
        if (val_lo.get())
            PB_CUDA_CHECK(cudaMemsetAsync(val_lo.get() + nnz, 0, size_t(nnz_pad - nnz) * 4, st));
    }
    tile_row_kernel<<<grid_1d(num_tiles + 1), kThreads, 0, st>>>(row_ptr.get(), rows, num_tiles,
                                                                 kSpmvTile, tile_row.get());
    PB_CUDA_CHECK(cudaGetLastError());
    reset_counters(st);
    PB_CUDA_CHECK(cudaMemsetAsync(carry.get(), 0, carry.bytes(), st));
}

void CsrDevice::reset_counters(cudaStream_t st) {
    if (counter.get()) PB_CUDA_CHECK(cudaMemsetAsync(counter.get(), 0, counter.bytes(), st));
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

void csr_upload_f64(CsrDevice& A, int rows, int cols, int nnz, const int* h_row_ptr,
                    const int* h_col, const double* h_val, cudaStream_t st, int* d_flag) {
    A.allocate(rows, cols, nnz, /*lo=*/true);
    upload_structure(A, rows, cols, nnz, h_row_ptr, h_col, st, d_flag);
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
    if (nnz > 0)
        PB_CUDA_CHECK(cudaMemcpyAsync(A.val.get(), h_val, size_t(nnz) * 4, cudaMemcpyHostToDevice, st));
    A.finalize(st);
}

void csr_transpose(const CsrDevice& A, CsrDevice& AT, cudaStream_t st) {
    const int nnz = A.nnz;
    AT.allocate(A.cols, A.rows, nnz, A.has_lo);
    if (nnz == 0) {
        PB_CUDA_CHECK(cudaMemsetAsync(AT.row_ptr.get(), 0, (size_t(A.cols) + 1) * 4, st));
        AT.finalize(st);
        return;
    }
    DevBuf<int> row_of{size_t(nnz)}, keys_out{size_t(nnz)}, perm_in{size_t(nnz)},
        perm_out{size_t(nnz)};
    {
        long long warps = A.rows;
        long long threads = warps * 32;
        expand_rows_kernel<<<grid_1d(threads), kThreads, 0, st>>>(A.row_ptr.get(), A.rows,
                                                                 row_of.get());
        PB_CUDA_CHECK(cudaGetLastError());
        iota_kernel<<<grid_1d(nnz), kThreads, 0, st>>>(perm_in.get(), nnz);
        PB_CUDA_CHECK(cudaGetLastError());
    }
    int end_bit = 1;
    while (end_bit < 31 && (1LL << end_bit) < (long long)A.cols) ++end_bit;
    size_t temp_bytes = 0;
    PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(nullptr, temp_bytes, A.col.get(), keys_out.get(),
                                                  perm_in.get(), perm_out.get(), nnz, 0, end_bit, st));
    DevBuf<unsigned char> temp(temp_bytes > 0 ? temp_bytes : 1);
    PB_CUDA_CHECK(cub::DeviceRadixSort::SortPairs(temp.get(), temp_bytes, A.col.get(),
                                                  keys_out.get(), perm_in.get(), perm_out.get(),
                                                  nnz, 0, end_bit, st));
    keys_to_rowptr_kernel<<<grid_1d((long long)A.cols + 1), kThreads, 0, st>>>(
        keys_out.get(), nnz, A.cols, AT.row_ptr.get());
    PB_CUDA_CHECK(cudaGetLastError());
    permute_kernel<<<grid_1d(nnz), kThreads, 0, st>>>(
        perm_out.get(), row_of.get(), A.val.get(), A.has_lo ? A.val_lo.get() : nullptr, nnz,
        AT.col.get(), AT.val.get(), AT.has_lo ? AT.val_lo.get() : nullptr);
    PB_CUDA_CHECK(cudaGetLastError());
    AT.finalize(st);
    PB_CUDA_CHECK(cudaStreamSynchronize(st));   // temporaries are freed on return
}

}  // namespace pb
