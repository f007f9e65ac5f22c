// gnn.cu — the warm-start network: graph packing, tensor-core dense layers,
// gather aggregations, deterministic reductions, loss, backward and Adam.
// The network itself is documented in gnn.cuh.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>

#include "gnn.cuh"
#include "umma.cuh"

namespace pb {

using bf16 = __nv_bfloat16;

// ---------------------------------------------------------------------------
// Tensor maps
// ---------------------------------------------------------------------------
namespace {
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    if (!fn) throw CudaError("CUDA error in gnn.cu - cuTensorMapEncodeTiled is unavailable");
    return fn;
}
}  // namespace

CUtensorMap make_bf16_tile_map(const void* base, long long rows, int cols, int pitch_elems, int box_rows) {
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const cuuint64_t dims[2] = {cuuint64_t(cols), cuuint64_t(rows > 0 ? rows : 1)};
    const cuuint64_t strides[1] = {cuuint64_t(pitch_elems) * 2};
    const cuuint32_t box[2] = {64u, cuuint32_t(box_rows)};
    const cuuint32_t estr[2] = {1u, 1u};
    const CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box,
                                   estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        throw CudaError("CUDA error in gnn.cu - cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")");
    return m;
}

namespace {

constexpr int kT = 256;
int grid_for(long long work) {
    long long g = (work + kT - 1) / kT;
    return int(std::max<long long>(1, std::min<long long>(g, 148LL * 32)));
}
#define GNN_STRIDE(i, n) \
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < (n); i += (long long)gridDim.x * blockDim.x)

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float bfr(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// ---------------------------------------------------------------------------
// Dense layers on the tensor cores
// ---------------------------------------------------------------------------
constexpr int kRowsPerTile = 128;
constexpr uint32_t kBoxBytes = 128u * 128u;   // 128 rows x 64 BF16
constexpr int kDenseThreads = 128;

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Stores 32 consecutive FP32 values as BF16 (64 bytes).
__device__ __forceinline__ void store_bf16x32(bf16* dst, const float (&v)[32]) {
    uint4* d = reinterpret_cast<uint4*>(dst);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        uint32_t w[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            __nv_bfloat162 p = __floats2bfloat162_rn(v[8 * q + 2 * e], v[8 * q + 2 * e + 1]);
            w[e] = *reinterpret_cast<uint32_t*>(&p);
        }
        d[q] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}
__device__ __forceinline__ void store_f32x32(float* dst, const float (&v)[32]) {
    float4* d = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int q = 0; q < 8; ++q) d[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

// Waits, with a limit, for the TMA copies still in flight on a stage before
// the block exits after an error.
__device__ __forceinline__ void drain(uint64_t* bar, bool pending, uint32_t parity) {
    if (pending) mbar_wait_bounded(bar, parity);
}

// Forward: out[r][0:64] = bf16(relu(X[r] . W^T + b)), X = [rows][128] BF16.
// Shared memory: X stages 2 x 32 KB, W 16 KB, bias, barriers.
struct FwdSmem {
    static constexpr uint32_t kA = 0;
    static constexpr uint32_t kB = 2 * 2 * kBoxBytes;             // 65536
    static constexpr uint32_t kBias = kB + 2 * 64 * 128;          // 81920
    static constexpr uint32_t kBars = kBias + 64 * 4;
    static constexpr uint32_t kBytes = kBars + 64 + 1024;         // + alignment slack
};
constexpr uint32_t kIdescFwd = umma::idesc_bf16<128, 64, false, false>();
constexpr uint32_t kIdescDx = umma::idesc_bf16<128, 128, false, false>();
constexpr uint32_t kIdescDw = umma::idesc_bf16<128, 64, true, true>();

__global__ void __launch_bounds__(kDenseThreads) dense_fwd_kernel(const __grid_constant__ CUtensorMap map_x,
                                                                  const __grid_constant__ CUtensorMap map_w,
                                                                  const float* __restrict__ bias, bf16* __restrict__ out,
                                                                  int ld_out, int rows, int* status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = align1024(smem_raw);
    uint8_t* sA = sm + FwdSmem::kA;
    uint8_t* sB = sm + FwdSmem::kB;
    float* sbias = reinterpret_cast<float*>(sm + FwdSmem::kBias);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + FwdSmem::kBars);   // [2]
    uint64_t* wbar = full + 2;
    uint64_t* mbar = full + 3;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(full + 4);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ntiles = (rows + kRowsPerTile - 1) / kRowsPerTile;

    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(wbar, 1);
        mbar_init(mbar, 1);
        fence_mbar_init();
        umma::tma_prefetch_map(&map_x);
        umma::tma_prefetch_map(&map_w);
    }
    if (warp == 0) umma::tmem_alloc(tslot, 64);
    if (tid < 64) sbias[tid] = bias[tid];
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    bool pend[2] = {false, false};
    uint32_t uses[2] = {0, 0};
    if (tid == 0) {
        mbar_arrive_expect_tx(wbar, 2 * 64 * 128);
        umma::tma_load_2d(sB, &map_w, 0, 0, wbar);
        umma::tma_load_2d(sB + 64 * 128, &map_w, 64, 0, wbar);
        if (int(blockIdx.x) < ntiles) {
            mbar_arrive_expect_tx(&full[0], 2 * kBoxBytes);
            umma::tma_load_2d(sA, &map_x, 0, blockIdx.x * kRowsPerTile, &full[0]);
            umma::tma_load_2d(sA + kBoxBytes, &map_x, 64, blockIdx.x * kRowsPerTile, &full[0]);
            pend[0] = true;
        }
    }
    bool ok = true;
    bool w_pending = tid == 0;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int s = it & 1;
        if (tid == 0) {
            const int next = tile + gridDim.x;
            if (next < ntiles) {
                uint8_t* dst = sA + (s ^ 1) * 2 * kBoxBytes;
                mbar_arrive_expect_tx(&full[s ^ 1], 2 * kBoxBytes);
                umma::tma_load_2d(dst, &map_x, 0, next * kRowsPerTile, &full[s ^ 1]);
                umma::tma_load_2d(dst + kBoxBytes, &map_x, 64, next * kRowsPerTile, &full[s ^ 1]);
                pend[s ^ 1] = true;
            }
            bool w_ok = true;
            if (w_pending) { w_ok = mbar_wait_bounded(wbar, 0); w_pending = !w_ok; }
            const bool f_ok = w_ok && mbar_wait_bounded(&full[s], uses[s] & 1);
            if (f_ok) {
                pend[s] = false;
                ++uses[s];
                umma::fence_after_sync();
                const uint32_t a0 = smem_u32(sA + s * 2 * kBoxBytes), b0 = smem_u32(sB);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const uint64_t ad = umma::smem_desc(a0 + (k >> 2) * kBoxBytes + (k & 3) * 32, 16, 1024);
                    const uint64_t bd = umma::smem_desc(b0 + (k >> 2) * (64 * 128) + (k & 3) * 32, 16, 1024);
                    umma::mma_bf16(tmem, ad, bd, kIdescFwd, k > 0 ? 1u : 0u);
                }
                umma::mma_commit(mbar);
            } else {
                ok = false;
            }
        }
        ok = mbar_wait_bounded(mbar, it & 1) && ok;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        umma::fence_after_sync();
        __syncwarp();
        const int row = tile * kRowsPerTile + tid;
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            umma::tmem_ld32(taddr + h * 32, v);
#pragma unroll
            for (int c = 0; c < 32; ++c) v[c] = fmaxf(v[c] + sbias[h * 32 + c], 0.0f);
            if (row < rows) store_bf16x32(out + size_t(row) * ld_out + h * 32, v);
        }
        umma::fence_before_sync();
        __syncthreads();
    }
    if (tid == 0) {
        if (w_pending) mbar_wait_bounded(wbar, 0);   // a block without tiles still loaded W
        if (!ok) {
            atomicOr(status, kDevErrTimeout);
            drain(&full[0], pend[0], uses[0] & 1);
            drain(&full[1], pend[1], uses[1] & 1);
        }
    }
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 64);
    }
}

// Input gradient: [dh_prev | dagg][r] = dZ[r] . W  (dZ [rows][64] BF16,
// W^T given as [128][64] BF16), FP32 outputs of 64 columns each.
struct DxSmem {
    static constexpr uint32_t kA = 0;                      // 2 stages x 16 KB
    static constexpr uint32_t kB = 2 * kBoxBytes;          // W^T 16 KB
    static constexpr uint32_t kBars = kB + kBoxBytes;
    // padded so that at most four blocks (4 x 128 tensor-memory columns) share an SM
    static constexpr uint32_t kBytes = 57 * 1024;
};

__global__ void __launch_bounds__(kDenseThreads) dense_dx_kernel(const __grid_constant__ CUtensorMap map_dz,
                                                                 const __grid_constant__ CUtensorMap map_wt,
                                                                 float* __restrict__ dh_prev, float* __restrict__ dagg,
                                                                 int rows, int* status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = align1024(smem_raw);
    uint8_t* sA = sm + DxSmem::kA;
    uint8_t* sB = sm + DxSmem::kB;
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + DxSmem::kBars);
    uint64_t* wbar = full + 2;
    uint64_t* mbar = full + 3;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(full + 4);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ntiles = (rows + kRowsPerTile - 1) / kRowsPerTile;

    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        mbar_init(wbar, 1);
        mbar_init(mbar, 1);
        fence_mbar_init();
        umma::tma_prefetch_map(&map_dz);
        umma::tma_prefetch_map(&map_wt);
    }
    if (warp == 0) umma::tmem_alloc(tslot, 128);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    bool pend[2] = {false, false};
    uint32_t uses[2] = {0, 0};
    if (tid == 0) {
        mbar_arrive_expect_tx(wbar, kBoxBytes);
        umma::tma_load_2d(sB, &map_wt, 0, 0, wbar);
        if (int(blockIdx.x) < ntiles) {
            mbar_arrive_expect_tx(&full[0], kBoxBytes);
            umma::tma_load_2d(sA, &map_dz, 0, blockIdx.x * kRowsPerTile, &full[0]);
            pend[0] = true;
        }
    }
    bool ok = true;
    bool w_pending = tid == 0;
    int it = 0;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++it) {
        const int s = it & 1;
        if (tid == 0) {
            const int next = tile + gridDim.x;
            if (next < ntiles) {
                mbar_arrive_expect_tx(&full[s ^ 1], kBoxBytes);
                umma::tma_load_2d(sA + (s ^ 1) * kBoxBytes, &map_dz, 0, next * kRowsPerTile, &full[s ^ 1]);
                pend[s ^ 1] = true;
            }
            bool w_ok = true;
            if (w_pending) { w_ok = mbar_wait_bounded(wbar, 0); w_pending = !w_ok; }
            const bool f_ok = w_ok && mbar_wait_bounded(&full[s], uses[s] & 1);
            if (f_ok) {
                pend[s] = false;
                ++uses[s];
                umma::fence_after_sync();
                const uint32_t a0 = smem_u32(sA + s * kBoxBytes), b0 = smem_u32(sB);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const uint64_t ad = umma::smem_desc(a0 + k * 32, 16, 1024);
                    const uint64_t bd = umma::smem_desc(b0 + k * 32, 16, 1024);
                    umma::mma_bf16(tmem, ad, bd, kIdescDx, k > 0 ? 1u : 0u);
                }
                umma::mma_commit(mbar);
            } else {
                ok = false;
            }
        }
        ok = mbar_wait_bounded(mbar, it & 1) && ok;
        if (!__syncthreads_and(ok)) { ok = false; break; }
        umma::fence_after_sync();
        __syncwarp();
        const int row = tile * kRowsPerTile + tid;
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16);
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            float v[32];
            umma::tmem_ld32(taddr + h * 32, v);
            if (row < rows) {
                float* dst = h < 2 ? dh_prev + size_t(row) * 64 + h * 32 : dagg + size_t(row) * 64 + (h - 2) * 32;
                store_f32x32(dst, v);
            }
        }
        umma::fence_before_sync();
        __syncthreads();
    }
    if (tid == 0) {
        if (w_pending) mbar_wait_bounded(wbar, 0);   // a block without tiles still loaded W
        if (!ok) {
            atomicOr(status, kDevErrTimeout);
            drain(&full[0], pend[0], uses[0] & 1);
            drain(&full[1], pend[1], uses[1] & 1);
        }
    }
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 128);
    }
}

// Weight gradient: partial[block][f][g] = sum over this block's row tiles of
// X[r][f] dZ[r][g]  (D = X^T dZ, both operands MN-major, K = rows).
struct DwSmem {
    static constexpr uint32_t kStage = 3 * kBoxBytes;      // X (2 boxes) + dZ (1 box)
    static constexpr uint32_t kBars = 2 * kStage;          // 98304
    static constexpr uint32_t kBytes = kBars + 64 + 1024;
};

__global__ void __launch_bounds__(kDenseThreads) dense_dw_kernel(const __grid_constant__ CUtensorMap map_x,
                                                                 const __grid_constant__ CUtensorMap map_dz,
                                                                 float* __restrict__ partial, int rows, int* status) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* sm = align1024(smem_raw);
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + DwSmem::kBars);   // [2]
    uint64_t* empty = full + 2;                                          // [2]
    uint64_t* done = full + 4;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(full + 5);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int ntiles = (rows + kRowsPerTile - 1) / kRowsPerTile;
    const int mine = ntiles > int(blockIdx.x) ? (ntiles - 1 - int(blockIdx.x)) / int(gridDim.x) + 1 : 0;

    if (tid == 0) {
        for (int i = 0; i < 5; ++i) mbar_init(&full[i], 1);
        fence_mbar_init();
        umma::tma_prefetch_map(&map_x);
        umma::tma_prefetch_map(&map_dz);
    }
    if (warp == 0) umma::tmem_alloc(tslot, 64);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = *tslot;

    bool ok = true;
    if (tid == 0) {
        bool pend[2] = {false, false};
        uint32_t fuses[2] = {0, 0}, euses[2] = {0, 0};
        auto load = [&](int i) {
            const int s = i & 1;
            const int r0 = (int(blockIdx.x) + i * int(gridDim.x)) * kRowsPerTile;
            uint8_t* st = sm + s * DwSmem::kStage;
            mbar_arrive_expect_tx(&full[s], 3 * kBoxBytes);
            umma::tma_load_2d(st, &map_x, 0, r0, &full[s]);
            umma::tma_load_2d(st + kBoxBytes, &map_x, 64, r0, &full[s]);
            umma::tma_load_2d(st + 2 * kBoxBytes, &map_dz, 0, r0, &full[s]);
            pend[s] = true;
        };
        if (mine > 0) load(0);
        if (mine > 1) load(1);
        for (int i = 0; i < mine; ++i) {
            const int s = i & 1;
            if (!mbar_wait_bounded(&full[s], fuses[s] & 1)) { ok = false; break; }
            pend[s] = false;
            ++fuses[s];
            umma::fence_after_sync();
            const uint32_t a0 = smem_u32(sm + s * DwSmem::kStage);
            const uint32_t b0 = a0 + 2 * kBoxBytes;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                // A: two 64-feature chunks 16 KB apart (LBO); B: one 64-wide chunk, so its
                // LBO is unused and kept small (every address stays inside this stage)
                const uint64_t ad = umma::smem_desc(a0 + k * 2048, kBoxBytes, 1024);
                const uint64_t bd = umma::smem_desc(b0 + k * 2048, 1024, 1024);
                umma::mma_bf16(tmem, ad, bd, kIdescDw, (i > 0 || k > 0) ? 1u : 0u);
            }
            umma::mma_commit(&empty[s]);
            if (i + 2 < mine) {
                if (!mbar_wait_bounded(&empty[s], euses[s] & 1)) { ok = false; break; }
                ++euses[s];
                load(i + 2);
            }
        }
        umma::mma_commit(done);
        if (!ok) {
            atomicOr(status, kDevErrTimeout);
            drain(&full[0], pend[0], fuses[0] & 1);
            drain(&full[1], pend[1], fuses[1] & 1);
        }
    }
    ok = mbar_wait_bounded(done, 0) && ok;
    ok = __syncthreads_and(ok);
    umma::fence_after_sync();
    __syncwarp();
    if (ok && mine > 0) {
        const uint32_t taddr = tmem + (uint32_t(warp * 32) << 16);
        float* dst = partial + (size_t(blockIdx.x) * 128 + tid) * 64;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            float v[32];
            umma::tmem_ld32(taddr + h * 32, v);
            store_f32x32(dst + h * 32, v);
        }
    } else if (mine == 0) {
        float* dst = partial + (size_t(blockIdx.x) * 128 + tid) * 64;
        for (int c = 0; c < 64; ++c) dst[c] = 0.0f;
    }
    if (!ok && tid == 0) atomicOr(status, kDevErrTimeout);
    umma::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        umma::fence_after_sync();
        umma::tmem_dealloc(tmem, 64);
    }
}

// dW[g][f] = sum_b partial[b][f][g], blocks in order.
__global__ void dw_reduce_kernel(const float* __restrict__ partial, int blocks, float* __restrict__ dw) {
    GNN_STRIDE(t, 64 * 128) {
        const int g = int(t / 128), f = int(t % 128);
        float acc = 0.0f;
        for (int b = 0; b < blocks; ++b) acc += partial[(size_t(b) * 128 + f) * 64 + g];
        dw[t] = acc;
    }
}

// ---------------------------------------------------------------------------
// CUDA-core kernels
// ---------------------------------------------------------------------------
// h0[r][o] = bf16(relu(sum_f W[o][f] feat[r][f] + b[o]))
constexpr int kF = kGnnFeat;
__global__ void input_layer_kernel(const float* __restrict__ feat, int nodes, const float* __restrict__ w,
                                   bf16* __restrict__ out, int ld) {
    __shared__ float sw[64 * kF + 64];
    for (int t = threadIdx.x; t < 64 * kF + 64; t += blockDim.x) sw[t] = w[t];
    __syncthreads();
    GNN_STRIDE(t, (long long)nodes * 64) {
        const long long r = t >> 6;
        const int o = int(t & 63);
        const float* f = feat + r * kF;
        float acc = 0.0f;
#pragma unroll
        for (int q = 0; q < kF; ++q) acc = fmaf(sw[o * kF + q], f[q], acc);
        acc += sw[64 * kF + o];
        out[r * ld + o] = __float2bfloat16_rn(fmaxf(acc, 0.0f));
    }
}

// out[r][64:128] = bf16(sum_{e in row r} coef[e] h[col[e]][0:64]); one warp per row.
__global__ void aggregate_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                 const float* __restrict__ coef, const bf16* __restrict__ h, int ldh,
                                 bf16* __restrict__ out, int ldo, int rows) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
        const int beg = rp[r], end = rp[r + 1];
        float a0 = 0.0f, a1 = 0.0f;
        for (int base = beg; base < end; base += 32) {
            const int e = base + lane;
            const int c = e < end ? col[e] : 0;
            const float w = e < end ? coef[e] : 0.0f;
            const int cnt = min(32, end - base);
            for (int t = 0; t < cnt; ++t) {
                const int cc = __shfl_sync(0xffffffffu, c, t);
                const float ww = __shfl_sync(0xffffffffu, w, t);
                const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(h + size_t(cc) * ldh + 2 * lane);
                a0 = fmaf(ww, __low2float(v), a0);
                a1 = fmaf(ww, __high2float(v), a1);
            }
        }
        *reinterpret_cast<__nv_bfloat162*>(out + size_t(r) * ldo + 64 + 2 * lane) = __floats2bfloat162_rn(a0, a1);
    }
}

// dh[r][0:64] += sum_{e in row r} coef[e] dagg[col[e]][0:64] (FP32).
__global__ void aggregate_bwd_kernel(const int* __restrict__ rp, const int* __restrict__ col,
                                     const float* __restrict__ coef, const float* __restrict__ dagg,
                                     float* __restrict__ dh, int rows) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < rows; r += warps) {
        const int beg = rp[r], end = rp[r + 1];
        float a0 = 0.0f, a1 = 0.0f;
        for (int base = beg; base < end; base += 32) {
            const int e = base + lane;
            const int c = e < end ? col[e] : 0;
            const float w = e < end ? coef[e] : 0.0f;
            const int cnt = min(32, end - base);
            for (int t = 0; t < cnt; ++t) {
                const int cc = __shfl_sync(0xffffffffu, c, t);
                const float ww = __shfl_sync(0xffffffffu, w, t);
                const float2 v = *reinterpret_cast<const float2*>(dagg + size_t(cc) * 64 + 2 * lane);
                a0 = fmaf(ww, v.x, a0);
                a1 = fmaf(ww, v.y, a1);
            }
        }
        float2* d = reinterpret_cast<float2*>(dh + size_t(r) * 64 + 2 * lane);
        float2 o = *d;
        o.x += a0;
        o.y += a1;
        *d = o;
    }
}

// out[r] = base[r] + (w . h[r] + b) (w: 64 rounded weights, then the bias); one warp per node.
__global__ void head_kernel(const bf16* __restrict__ h, int nodes, const float* __restrict__ wb,
                            const float* __restrict__ base, float* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long r = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; r < nodes; r += warps) {
        const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(h + size_t(r) * 64 + 2 * lane);
        float p = fmaf(wb[2 * lane + 1], __high2float(v), wb[2 * lane] * __low2float(v));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0) out[r] = base[r] + (p + wb[64]);
    }
}

// Sums over the nodes of each chunk: part[c][t] = sum_{r in chunk c} F(r, t).
template <class F>
__global__ void chunk_kernel(F f, int width, const int* __restrict__ begin, int chunks, float* __restrict__ part) {
    for (int c = blockIdx.x; c < chunks; c += gridDim.x) {
        const int b = begin[c], e = begin[c + 1];
        for (int t = threadIdx.x; t < width; t += blockDim.x) {
            float acc = 0.0f;
            for (int r = b; r < e; ++r) acc += f(r, t);
            part[size_t(c) * width + t] = acc;
        }
    }
}

struct PoolF {          // h [r][64] BF16
    const bf16* h;
    __device__ float operator()(int r, int t) const { return bf(h[size_t(r) * 64 + t]); }
};
struct SqErrF {         // (hat - target)^2 / count of the node's LP
    const float* hat;
    const float* tgt;
    const int* lp;
    const float* inv;
    __device__ float operator()(int r, int) const {
        const float d = hat[r] - tgt[r];
        return d * d * inv[lp[r]];
    }
};
struct HeadGradF {      // t < 64: d[r] h[r][t]; t == 64: d[r]
    const bf16* h;
    const float* d;
    __device__ float operator()(int r, int t) const { return t < 64 ? d[r] * bf(h[size_t(r) * 64 + t]) : d[r]; }
};
struct BiasGradF {      // dz [r][64] BF16
    const bf16* dz;
    __device__ float operator()(int r, int t) const { return bf(dz[size_t(r) * 64 + t]); }
};
constexpr int kInW = 64 * kF;   // input-layer weights; the 64 biases follow
constexpr int kWide = kInW + 64; // widest chunk partial

// Input-layer gradient partials: part[c][o*9 + q] = sum_{r in chunk c} dz0[r][o] f[r][q],
// part[c][kInW + o] = sum_r dz0[r][o], with dz0 = dh0 masked by h0 > 0.  One
// thread per output feature o (coalesced dh / h0 reads), nodes in order.
__global__ void inlayer_grad_kernel(const float* __restrict__ dh, const bf16* __restrict__ h0, int ldh0,
                                    const float* __restrict__ feat, const int* __restrict__ begin, int chunks,
                                    float* __restrict__ part) {
    const int o = threadIdx.x;   // blockDim.x == 64
    for (int c = blockIdx.x; c < chunks; c += gridDim.x) {
        float acc[kF + 1];
#pragma unroll
        for (int q = 0; q <= kF; ++q) acc[q] = 0.0f;
        for (int r = begin[c]; r < begin[c + 1]; ++r) {
            const float g = bf(h0[size_t(r) * ldh0 + o]) > 0.0f ? dh[size_t(r) * 64 + o] : 0.0f;
            const float* f = feat + size_t(r) * kF;
#pragma unroll
            for (int q = 0; q < kF; ++q) acc[q] += g * f[q];
            acc[kF] += g;
        }
        float* dst = part + size_t(c) * kWide;
#pragma unroll
        for (int q = 0; q < kF; ++q) dst[o * kF + q] = acc[q];
        dst[kInW + o] = acc[kF];
    }
}

// out[k][t] = scale_k * sum_{c in LP k's chunks} part[c][t]
__global__ void lp_sum_kernel(const float* __restrict__ part, int width, const int* __restrict__ lp_first, int K,
                              const float* __restrict__ inv, float* __restrict__ out, int ld_out) {
    GNN_STRIDE(t, (long long)K * width) {
        const int k = int(t / width), w = int(t % width);
        float acc = 0.0f;
        for (int c = lp_first[k]; c < lp_first[k + 1]; ++c) acc += part[size_t(c) * width + w];
        out[size_t(k) * ld_out + w] = inv ? acc * inv[k] : acc;
    }
}

// Ordered group sums: dst[g][t] = sum_{r in [64g, 64g+64)} src[r][t].
__global__ void group_sum_kernel(const float* __restrict__ src, int rows, int width, float* __restrict__ dst) {
    const int groups = (rows + 63) / 64;
    GNN_STRIDE(t, (long long)groups * width) {
        const int g = int(t / width), w = int(t % width);
        float acc = 0.0f;
        const int e = min(rows, 64 * g + 64);
        for (int r = 64 * g; r < e; ++r) acc += src[size_t(r) * width + w];
        dst[t] = acc;
    }
}

// rho_k = w_w . pooled_k + b_w (128 weights, then the bias); one warp per LP.
__global__ void rho_kernel(const float* __restrict__ pooled, int K, const float* __restrict__ wb,
                           float* __restrict__ rho) {
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long k = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5; k < K; k += warps) {
        float p = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) p = fmaf(wb[4 * lane + q], pooled[size_t(k) * 128 + 4 * lane + q], p);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
        if (lane == 0) rho[k] = p + wb[128];
    }
}

// d[r] = 2 (hat[r] - tgt[r]) inv[lp[r]] / K
__global__ void head_delta_kernel(const float* __restrict__ hat, const float* __restrict__ tgt,
                                  const int* __restrict__ lp, const float* __restrict__ inv, float inv_k, int nodes,
                                  float* __restrict__ d) {
    GNN_STRIDE(r, nodes) d[r] = 2.0f * (hat[r] - tgt[r]) * inv[lp[r]] * inv_k;
}

// dh[r][f] = d[r] w[f] + drho[lp] ww[f] inv[lp]
__global__ void head_back_kernel(const float* __restrict__ d, const int* __restrict__ lp, const float* __restrict__ w,
                                 const float* __restrict__ drho, const float* __restrict__ ww,
                                 const float* __restrict__ inv, int nodes, float* __restrict__ dh) {
    GNN_STRIDE(t, (long long)nodes * 64) {
        const long long r = t >> 6;
        const int f = int(t & 63);
        const int k = lp[r];
        dh[t] = fmaf(d[r], w[f], drho[k] * ww[f] * inv[k]);
    }
}

// out[t] = sum_k drho[k] pooled[k][t] (t < 128), sum_k drho[k] (t = 128); LPs in order.
__global__ void rho_grad_kernel(const float* __restrict__ pooled, const float* __restrict__ drho, int K,
                                float* __restrict__ out) {
    for (int t = threadIdx.x; t < 129; t += blockDim.x) {
        float acc = 0.0f;
        for (int k = 0; k < K; ++k) acc += t < 128 ? drho[k] * pooled[size_t(k) * 128 + t] : drho[k];
        out[t] = acc;
    }
}

// dz[r][f] = bf16(h[r][f] > 0 ? dh[r][f] : 0)
__global__ void dz_kernel(const float* __restrict__ dh, const bf16* __restrict__ h, int ldh, int nodes,
                          bf16* __restrict__ dz) {
    GNN_STRIDE(t, (long long)nodes * 64) {
        const long long r = t >> 6;
        const int f = int(t & 63);
        dz[t] = __float2bfloat16_rn(bf(h[r * ldh + f]) > 0.0f ? dh[t] : 0.0f);
    }
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, int n, float lr, float c1, float c2) {
    constexpr float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    GNN_STRIDE(i, n) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
    }
}

// pr = bf16-rounded parameters; w / wt = the dense layers' W and W^T in BF16.
__global__ void refresh_kernel(const float* __restrict__ p, int n, float* __restrict__ pr, bf16* __restrict__ w,
                               bf16* __restrict__ wt) {
    GNN_STRIDE(i, n) pr[i] = bfr(p[i]);
    GNN_STRIDE(t, 2LL * kGnnLayers * 64 * 128) {
        const int d = int(t / (64 * 128)), e = int(t % (64 * 128));
        const int l = d >> 1, side = d & 1;
        const int g = e / 128, f = e % 128;
        const bf16 v = __float2bfloat16_rn(p[GnnParams::layer_w(l, side) + e]);
        w[t] = v;
        wt[size_t(d) * 64 * 128 + size_t(f) * 64 + g] = v;
    }
}

// splitmix64 uniform in [-a, a)
uint64_t splitmix(uint64_t& s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
float uniform(uint64_t& s, float a) {
    const double u = double(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
    return float((2.0 * u - 1.0) * a);
}

int dense_blocks(int dev, int rows, int per_sm) {
    const int tiles = (rows + kRowsPerTile - 1) / kRowsPerTile;
    return std::max(1, std::min(tiles, per_sm * device_sm_count(dev)));
}

void set_smem_attrs_once() {
    static std::once_flag once;
    std::call_once(once, [] {
        PB_CUDA_CHECK(cudaFuncSetAttribute(dense_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(FwdSmem::kBytes)));
        PB_CUDA_CHECK(cudaFuncSetAttribute(dense_dx_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(DxSmem::kBytes)));
        PB_CUDA_CHECK(cudaFuncSetAttribute(dense_dw_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(DwSmem::kBytes)));
    });
}

}  // namespace

// ---------------------------------------------------------------------------
// GnnGraph
// ---------------------------------------------------------------------------
GnnGraph::GnnGraph(const pramaan_lp* lps, int count_, const pramaan_warm_start* hints,
                   const pramaan_warm_start* targets, int dev) {
    device = dev;
    count = count_;
    has_targets = targets != nullptr;
    long long M = 0, N = 0, NZ = 0;
    for (int k = 0; k < count; ++k) {
        const pramaan_lp& lp = lps[k];
        if (lp.num_rows < 0 || lp.num_cols < 0 || lp.nnz < 0) throw InvalidArgument("gnn graph: negative size");
        if (lp.num_cols == 0) continue;
        index.push_back(k);
        r0.push_back(int(M));
        c0.push_back(int(N));
        M += lp.num_rows;
        N += lp.num_cols;
        NZ += lp.nnz;
        if (M > INT_MAX / 2 || N > INT_MAX / 2 || NZ > INT_MAX / 2)
            throw InvalidArgument("gnn graph: the packed batch exceeds 2^30 rows, columns or non-zeros");
    }
    K = int(index.size());
    m = int(M);
    n = int(N);
    nnz = int(NZ);
    r0.push_back(m);
    c0.push_back(n);
    PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (K == 0) return;

    const size_t Mz = static_cast<size_t>(m), Nz = static_cast<size_t>(n), Ez = static_cast<size_t>(nnz);
    std::vector<int> hrp(Mz + 1, 0), hci(Ez), hlpr(Mz), hlpc(Nz);
    std::vector<double> hval(Ez), hvlo(Nz), hvhi(Nz), hcost(Nz), hrlo(Mz), hrhi(Mz);
    s_a.assign(size_t(K), 1.0);
    s_b.assign(size_t(K), 1.0);
    s_c.assign(size_t(K), 1.0);
    omega_ref.assign(size_t(K), 1.0);
    long long e0 = 0;
    for (int q = 0; q < K; ++q) {
        const pramaan_lp& lp = lps[index[size_t(q)]];
        if (lp.num_rows > 0 && !lp.row_ptr) throw InvalidArgument("gnn graph: row_ptr is NULL");
        if (lp.nnz > 0 && (!lp.col_idx || !lp.values)) throw InvalidArgument("gnn graph: col_idx/values is NULL");
        if (!lp.obj_coeffs || !lp.var_lower || !lp.var_upper) throw InvalidArgument("gnn graph: column data is NULL");
        if (lp.num_rows > 0 && (!lp.row_lower || !lp.row_upper)) throw InvalidArgument("gnn graph: row bounds are NULL");
        if (lp.num_rows > 0 && (lp.row_ptr[0] != 0 || lp.row_ptr[lp.num_rows] != lp.nnz))
            throw InvalidArgument("pramaan_lp: row_ptr must start at 0, be non-decreasing and end at nnz");
        const double sign = lp.obj_sense == PRAMAAN_MAXIMIZE ? -1.0 : 1.0;
        const int R = r0[size_t(q)], C = c0[size_t(q)];
        double a2 = 0.0, b2 = 0.0, c2 = 0.0;
        long long bc = 0;
        for (int i = 0; i < lp.num_rows; ++i) {
            if (lp.row_ptr[i + 1] < lp.row_ptr[i]) throw InvalidArgument("pramaan_lp: row_ptr must be non-decreasing");
            hrp[size_t(R + i)] = int(e0 + lp.row_ptr[i]);
            hlpr[size_t(R + i)] = q;
            const double lo = lp.row_lower[i], hi = lp.row_upper[i];
            hrlo[size_t(R + i)] = lo;
            hrhi[size_t(R + i)] = hi;
            if (lo > -1e29) { b2 += lo * lo; ++bc; }
            if (hi < 1e29 && !(lo > -1e29 && lo == hi)) { b2 += hi * hi; ++bc; }
        }
        for (int e = 0; e < lp.nnz; ++e) {
            const int j = lp.col_idx[e];
            if (j < 0 || j >= lp.num_cols) throw InvalidArgument("pramaan_lp: col_idx entry out of bounds");
            hci[size_t(e0 + e)] = C + j;
            hval[size_t(e0 + e)] = lp.values[e];
            a2 += lp.values[e] * lp.values[e];
        }
        for (int j = 0; j < lp.num_cols; ++j) {
            const double cj = sign * lp.obj_coeffs[j];
            hcost[size_t(C + j)] = cj;
            c2 += cj * cj;
            hvlo[size_t(C + j)] = lp.var_lower[j];
            hvhi[size_t(C + j)] = lp.var_upper[j];
            hlpc[size_t(C + j)] = q;
        }
        e0 += lp.nnz;
        const double sa = lp.nnz > 0 ? std::sqrt(a2 / lp.nnz) : 0.0;
        const double sb = bc > 0 ? std::sqrt(b2 / double(bc)) : 0.0;
        const double sc = std::sqrt(c2 / lp.num_cols);
        s_a[size_t(q)] = sa > 0.0 && std::isfinite(sa) ? sa : 1.0;
        s_b[size_t(q)] = sb > 0.0 && std::isfinite(sb) ? sb : 1.0;
        s_c[size_t(q)] = sc > 0.0 && std::isfinite(sc) ? sc : 1.0;
        const double cn = std::sqrt(c2), bn = std::sqrt(b2);
        omega_ref[size_t(q)] = cn > 1e-10 && bn > 1e-10 && std::isfinite(cn / bn) ? cn / bn : 1.0;
    }
    hrp[size_t(m)] = int(e0);

    // transpose (counting sort by column; rows of A^T list A's rows in order)
    std::vector<int> deg_c(Nz, 0), htp(Nz + 1, 0), hti(Ez), perm(Ez);
    for (int e = 0; e < nnz; ++e) ++deg_c[size_t(hci[size_t(e)])];
    for (int j = 0; j < n; ++j) htp[size_t(j) + 1] = htp[size_t(j)] + deg_c[size_t(j)];
    {
        std::vector<int> pos(htp.begin(), htp.end() - 1);
        for (int i = 0; i < m; ++i)
            for (int e = hrp[size_t(i)]; e < hrp[size_t(i) + 1]; ++e) {
                const int p = pos[size_t(hci[size_t(e)])]++;
                hti[size_t(p)] = i;
                perm[size_t(p)] = e;
            }
    }
    std::vector<float> hcr(Ez), hcc(Ez), htr(Ez), htc(Ez);
    for (int i = 0; i < m; ++i) {
        const int q = hlpr[size_t(i)];
        const int deg = hrp[size_t(i) + 1] - hrp[size_t(i)];
        for (int e = hrp[size_t(i)]; e < hrp[size_t(i) + 1]; ++e) {
            const int j = hci[size_t(e)];
            hcr[size_t(e)] = float(hval[size_t(e)] / (s_a[size_t(q)] * std::max(1, deg)));
            hcc[size_t(e)] = float(hval[size_t(e)] / (s_a[size_t(q)] * std::max(1, deg_c[size_t(j)])));
        }
    }
    for (int p = 0; p < nnz; ++p) {
        htr[size_t(p)] = hcr[size_t(perm[size_t(p)])];
        htc[size_t(p)] = hcc[size_t(perm[size_t(p)])];
    }

    // features (FP64 arithmetic, stored as FP32)
    auto clip = [](double v) { return std::min(10.0, std::max(-10.0, v)); };
    std::vector<float> hfv(Nz * kF), hfc(Mz * kF), hbx(Nz, 0.0f), hby(Mz, 0.0f);
    std::vector<char> hint_x(Nz, 0), hint_y(Mz, 0);
    if (hints) {
        for (int q = 0; q < K; ++q) {
            const pramaan_warm_start& h = hints[index[size_t(q)]];
            const int C = c0[size_t(q)], R = r0[size_t(q)];
            const int nk = c0[size_t(q) + 1] - C, mk = r0[size_t(q) + 1] - R;
            const double sa = s_a[size_t(q)], sb = s_b[size_t(q)], sc = s_c[size_t(q)];
            if (h.x)
                for (int j = 0; j < nk; ++j) {
                    if (!std::isfinite(h.x[j])) throw InvalidArgument("gnn graph: hint x must be finite");
                    hbx[size_t(C + j)] = float(h.x[j] * sa / sb);
                    hint_x[size_t(C + j)] = 1;
                }
            if (h.y)
                for (int i = 0; i < mk; ++i) {
                    if (!std::isfinite(h.y[i])) throw InvalidArgument("gnn graph: hint y must be finite");
                    hby[size_t(R + i)] = float(h.y[i] * sa / sc);
                    hint_y[size_t(R + i)] = 1;
                }
        }
    }
    for (int j = 0; j < n; ++j) {
        const int q = hlpc[size_t(j)];
        const double sa = s_a[size_t(q)], sb = s_b[size_t(q)], sc = s_c[size_t(q)];
        const double lo = hvlo[size_t(j)], hi = hvhi[size_t(j)];
        const bool fl = lo > -1e29, fu = hi < 1e29;
        double absum = 0.0;
        for (int p = htp[size_t(j)]; p < htp[size_t(j) + 1]; ++p) absum += std::fabs(hval[size_t(perm[size_t(p)])]);
        const int deg = deg_c[size_t(j)];
        float* f = &hfv[size_t(j) * kF];
        f[0] = float(hcost[size_t(j)] / sc);
        f[1] = fl ? 1.0f : 0.0f;
        f[2] = fu ? 1.0f : 0.0f;
        f[3] = fl ? float(clip(lo * sa / sb)) : 0.0f;
        f[4] = fu ? float(clip(hi * sa / sb)) : 0.0f;
        f[5] = float(std::log1p(double(deg)) / 4.0);
        f[6] = deg > 0 ? float(absum / (sa * deg)) : 0.0f;
        f[7] = hint_x[size_t(j)] ? 1.0f : 0.0f;
        f[8] = float(clip(double(hbx[size_t(j)])));
    }
    for (int i = 0; i < m; ++i) {
        const int q = hlpr[size_t(i)];
        const double sa = s_a[size_t(q)], sb = s_b[size_t(q)];
        const double lo = hrlo[size_t(i)], hi = hrhi[size_t(i)];
        const bool fl = lo > -1e29, fu = hi < 1e29;
        double absum = 0.0;
        for (int e = hrp[size_t(i)]; e < hrp[size_t(i) + 1]; ++e) absum += std::fabs(hval[size_t(e)]);
        const int deg = hrp[size_t(i) + 1] - hrp[size_t(i)];
        float* f = &hfc[size_t(i) * kF];
        f[0] = fl && fu && lo == hi ? 1.0f : 0.0f;
        f[1] = fl ? 1.0f : 0.0f;
        f[2] = fu ? 1.0f : 0.0f;
        f[3] = fl ? float(clip(lo / sb)) : 0.0f;
        f[4] = fu ? float(clip(hi / sb)) : 0.0f;
        f[5] = float(std::log1p(double(deg)) / 4.0);
        f[6] = deg > 0 ? float(absum / (sa * deg)) : 0.0f;
        f[7] = hint_y[size_t(i)] ? 1.0f : 0.0f;
        f[8] = float(clip(double(hby[size_t(i)])));
    }

    // chunk tables
    const size_t Kz = static_cast<size_t>(K);
    std::vector<int> cb, rb, clp, rlp, cfirst(Kz + 1), rfirst(Kz + 1);
    std::vector<float> hinv_n(Kz), hinv_m(Kz), hscale(Kz * 4);
    for (int q = 0; q < K; ++q) {
        cfirst[size_t(q)] = int(cb.size());
        for (int b = c0[size_t(q)]; b < c0[size_t(q) + 1]; b += kGnnChunk) { cb.push_back(b); clp.push_back(q); }
        rfirst[size_t(q)] = int(rb.size());
        for (int b = r0[size_t(q)]; b < r0[size_t(q) + 1]; b += kGnnChunk) { rb.push_back(b); rlp.push_back(q); }
        const int nk = c0[size_t(q) + 1] - c0[size_t(q)], mk = r0[size_t(q) + 1] - r0[size_t(q)];
        hinv_n[size_t(q)] = 1.0f / float(nk);
        hinv_m[size_t(q)] = mk > 0 ? 1.0f / float(mk) : 0.0f;
        hscale[size_t(q) * 4 + 0] = float(s_a[size_t(q)]);
        hscale[size_t(q) * 4 + 1] = float(s_b[size_t(q)]);
        hscale[size_t(q) * 4 + 2] = float(s_c[size_t(q)]);
        hscale[size_t(q) * 4 + 3] = 1.0f / float(K);
    }
    cfirst[size_t(K)] = int(cb.size());
    rfirst[size_t(K)] = int(rb.size());
    cchunks = int(cb.size());
    rchunks = int(rb.size());
    cb.push_back(n);
    rb.push_back(m);

    auto up = [&](auto& d, const auto& h) {
        d.alloc(h.size());
        if (!h.empty())
            PB_CUDA_CHECK(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(h[0]), cudaMemcpyHostToDevice, st));
    };
    up(rp, hrp); up(ci, hci); up(tp, htp); up(ti, hti);
    up(coef_r, hcr); up(coef_c, hcc); up(tcoef_r, htr); up(tcoef_c, htc);
    up(fv, hfv); up(fc, hfc); up(base_x, hbx); up(base_y, hby); up(lp_col, hlpc); up(lp_row, hlpr); up(lp_scale, hscale);
    up(vlo, hvlo); up(vhi, hvhi);
    up(cchunk_begin, cb); up(rchunk_begin, rb); up(cchunk_lp, clp); up(rchunk_lp, rlp);
    up(clp_first, cfirst); up(rlp_first, rfirst); up(inv_n, hinv_n); up(inv_m, hinv_m);
    h_vlo = std::move(hvlo);
    h_vhi = std::move(hvhi);

    if (has_targets) {
        std::vector<float> htx(Nz), hty(Mz), htw(Kz), hlx(Kz), hly(Kz);
        for (int q = 0; q < K; ++q) {
            const pramaan_warm_start& t = targets[index[size_t(q)]];
            const int nk = c0[size_t(q) + 1] - c0[size_t(q)], mk = r0[size_t(q) + 1] - r0[size_t(q)];
            if (!t.x || (mk > 0 && !t.y)) throw InvalidArgument("gnn graph: every target needs x (and y when m > 0)");
            if (!(t.primal_weight > 0.0) || !std::isfinite(t.primal_weight))
                throw InvalidArgument("gnn graph: target primal weights must be positive and finite");
            const double sa = s_a[size_t(q)], sb = s_b[size_t(q)], sc = s_c[size_t(q)];
            for (int j = 0; j < nk; ++j) htx[size_t(c0[size_t(q)] + j)] = float(t.x[j] * sa / sb);
            for (int i = 0; i < mk; ++i) hty[size_t(r0[size_t(q)] + i)] = float(t.y[i] * sa / sc);
            htw[size_t(q)] = float(std::log(t.primal_weight / omega_ref[size_t(q)]));
            // per-LP loss weights: squared errors relative to the mean square of the targets
            double sx = 0.0, sy = 0.0;
            for (int j = 0; j < nk; ++j) sx += double(htx[size_t(c0[size_t(q)] + j)]) * htx[size_t(c0[size_t(q)] + j)];
            for (int i = 0; i < mk; ++i) sy += double(hty[size_t(r0[size_t(q)] + i)]) * hty[size_t(r0[size_t(q)] + i)];
            hlx[size_t(q)] = float(1.0 / (nk * (sx / nk + kLossFloor)));
            hly[size_t(q)] = mk > 0 ? float(1.0 / (mk * (sy / mk + kLossFloor))) : 0.0f;
        }
        up(tx, htx); up(ty, hty); up(tw, htw); up(lw_x, hlx); up(lw_y, hly);
    }
    PB_CUDA_CHECK(cudaStreamSynchronize(st));
}

GnnGraph::~GnnGraph() {
    if (st) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
}

// ---------------------------------------------------------------------------
// GnnModel
// ---------------------------------------------------------------------------
GnnModel::GnnModel(int device, uint64_t seed) : dev_(device) {
    PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking));
    set_smem_attrs_once();
    const int np = GnnParams::kCount;
    p_.alloc(np); g_.alloc(np); am_.alloc(np); av_.alloc(np); pr_.alloc(np);
    w_.alloc(size_t(2 * kGnnLayers) * 64 * 128);
    wt_.alloc(size_t(2 * kGnnLayers) * 64 * 128);
    status_.alloc(1);
    // He-uniform weights (fan-in), zero biases and heads
    std::vector<float> h(size_t(np), 0.0f);
    uint64_t s = seed;
    auto fill = [&](int off, int count_, int fan_in) {
        const float a = std::sqrt(6.0f / float(fan_in));
        for (int i = 0; i < count_; ++i) h[size_t(off + i)] = uniform(s, a);
    };
    fill(GnnParams::kVinW, 64 * kGnnFeat, kGnnFeat);
    fill(GnnParams::kCinW, 64 * kGnnFeat, kGnnFeat);
    for (int l = 0; l < kGnnLayers; ++l)
        for (int side = 0; side < 2; ++side) fill(GnnParams::layer_w(l, side), 64 * 128, 128);
    // the heads start at zero: an untrained network returns the hint (or 0)
    // and omega_ref, and learns a correction from there
    set_params(h.data());
}

GnnModel::~GnnModel() {
    if (st_) {
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
}

void GnnModel::get_params(float* host) const {
    PB_CUDA_CHECK(cudaMemcpyAsync(host, p_.get(), p_.bytes(), cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

void GnnModel::set_params(const float* host) {
    PB_CUDA_CHECK(cudaMemcpyAsync(p_.get(), host, p_.bytes(), cudaMemcpyHostToDevice, st_));
    PB_CUDA_CHECK(cudaMemsetAsync(am_.get(), 0, am_.bytes(), st_));
    PB_CUDA_CHECK(cudaMemsetAsync(av_.get(), 0, av_.bytes(), st_));
    adam_t_ = 0;
    refresh_weights();
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

void GnnModel::refresh_weights() {
    refresh_kernel<<<grid_for(2LL * kGnnLayers * 64 * 128), kT, 0, st_>>>(p_.get(), GnnParams::kCount, pr_.get(),
                                                                         w_.get(), wt_.get());
    PB_CUDA_CHECK(cudaGetLastError());
}

void GnnModel::copy_grad(float* host) const {
    PB_CUDA_CHECK(cudaMemcpyAsync(host, g_.get(), g_.bytes(), cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

void GnnModel::ensure_workspace(const GnnGraph& g) {
    const size_t m = size_t(std::max(g.m, 1)), n = size_t(std::max(g.n, 1)), k = size_t(std::max(g.K, 1));
    const size_t chunks = size_t(std::max(std::max(g.cchunks, g.rchunks), 1));
    if (m > cap_m_) {
        for (auto& b : xc_) b.alloc(m * 128);
        hc3_.alloc(m * 64);
        dhc_.alloc(m * 64);
        yhat_.alloc(m);
        cap_m_ = m;
    }
    if (n > cap_n_) {
        for (auto& b : xv_) b.alloc(n * 128);
        hv3_.alloc(n * 64);
        dhv_.alloc(n * 64);
        xhat_.alloc(n);
        cap_n_ = n;
    }
    const size_t mx = std::max(cap_m_, cap_n_);
    if (dz_.size() < mx * 64) {
        dz_.alloc(mx * 64);
        dagg_.alloc(mx * 64);
    }
    if (k > cap_k_) {
        pooled_.alloc(k * 128);
        rho_.alloc(k * 4);         // rho, drho, loss_w, spare
        lp_sums_.alloc(k * 4);
        cap_k_ = k;
    }
    if (chunks > cap_chunks_) {
        // chunk partials and two ping-pong halves, up to kWide columns wide
        part_.alloc(chunks * kWide * 2 + kWide);
        cap_chunks_ = chunks;
    }
    if (wpart_.size() == 0) wpart_.alloc(size_t(2 * device_sm_count(dev_)) * 128 * 64);
}

namespace {
// Deterministic total over `rows` partial rows of `width` columns; the result
// lands in `out` (device).  `scratch` holds at least rows/64 + 1 rows.
void ordered_total(const float* part, int rows, int width, float* scratch, float* out, cudaStream_t st) {
    const float* cur = part;
    float* bufs[2] = {scratch, scratch + size_t((rows + 63) / 64 + 1) * width};
    int b = 0;
    while (rows > 1) {
        const int groups = (rows + 63) / 64;
        float* dst = groups == 1 ? out : bufs[b];
        group_sum_kernel<<<grid_for((long long)groups * width), kT, 0, st>>>(cur, rows, width, dst);
        PB_CUDA_CHECK(cudaGetLastError());
        cur = dst;
        rows = groups;
        b ^= 1;
    }
    if (rows == 1 && cur != out)
        PB_CUDA_CHECK(cudaMemcpyAsync(out, cur, size_t(width) * 4, cudaMemcpyDeviceToDevice, st));
}
}  // namespace

void GnnModel::forward(const GnnGraph& g) {
    last_ = &g;
    if (g.K == 0) return;
    ensure_workspace(g);
    PB_CUDA_CHECK(cudaMemsetAsync(status_.get(), 0, 4, st_));
    const float* pr = pr_.get();
    // input layers
    input_layer_kernel<<<grid_for((long long)g.n * 64), kT, 0, st_>>>(g.fv.get(), g.n, pr + GnnParams::kVinW,
                                                                      xv_[0].get(), 128);
    if (g.m > 0)
        input_layer_kernel<<<grid_for((long long)g.m * 64), kT, 0, st_>>>(g.fc.get(), g.m, pr + GnnParams::kCinW,
                                                                          xc_[0].get(), 128);
    PB_CUDA_CHECK(cudaGetLastError());
    for (int l = 0; l < kGnnLayers; ++l) {
        bf16* out_c = l + 1 < kGnnLayers ? xc_[l + 1].get() : hc3_.get();
        bf16* out_v = l + 1 < kGnnLayers ? xv_[l + 1].get() : hv3_.get();
        const int ldo = l + 1 < kGnnLayers ? 128 : 64;
        if (g.m > 0) {
            aggregate_kernel<<<grid_for((long long)g.m * 32), kT, 0, st_>>>(g.rp.get(), g.ci.get(), g.coef_r.get(),
                                                                            xv_[l].get(), 128, xc_[l].get(), 128, g.m);
            PB_CUDA_CHECK(cudaGetLastError());
            const CUtensorMap mx = make_bf16_tile_map(xc_[l].get(), g.m, 128, 128, 128);
            const CUtensorMap mw = make_bf16_tile_map(w_.get() + size_t(2 * l) * 64 * 128, 64, 128, 128, 64);
            dense_fwd_kernel<<<dense_blocks(dev_, g.m, 2), kDenseThreads, FwdSmem::kBytes, st_>>>(
                mx, mw, pr + GnnParams::layer_b(l, 0), out_c, ldo, g.m, status_.get());
            PB_CUDA_CHECK(cudaGetLastError());
            aggregate_kernel<<<grid_for((long long)g.n * 32), kT, 0, st_>>>(g.tp.get(), g.ti.get(), g.tcoef_c.get(),
                                                                            out_c, ldo, xv_[l].get(), 128, g.n);
        } else {
            // no constraints: the aggregated half of the variable input is zero
            PB_CUDA_CHECK(cudaMemset2DAsync(xv_[l].get() + 64, 256, 0, 128, size_t(g.n), st_));
        }
        PB_CUDA_CHECK(cudaGetLastError());
        const CUtensorMap mx = make_bf16_tile_map(xv_[l].get(), g.n, 128, 128, 128);
        const CUtensorMap mw = make_bf16_tile_map(w_.get() + size_t(2 * l + 1) * 64 * 128, 64, 128, 128, 64);
        dense_fwd_kernel<<<dense_blocks(dev_, g.n, 2), kDenseThreads, FwdSmem::kBytes, st_>>>(
            mx, mw, pr + GnnParams::layer_b(l, 1), out_v, ldo, g.n, status_.get());
        PB_CUDA_CHECK(cudaGetLastError());
    }
    // heads
    head_kernel<<<grid_for((long long)g.n * 32), kT, 0, st_>>>(hv3_.get(), g.n, pr + GnnParams::kHeadX,
                                                               g.base_x.get(), xhat_.get());
    if (g.m > 0)
        head_kernel<<<grid_for((long long)g.m * 32), kT, 0, st_>>>(hc3_.get(), g.m, pr + GnnParams::kHeadY,
                                                                   g.base_y.get(), yhat_.get());
    PB_CUDA_CHECK(cudaGetLastError());
    // pooled means per LP, then rho
    float* part = part_.get();
    chunk_kernel<<<std::min(g.cchunks, 148 * 8), 64, 0, st_>>>(PoolF{hv3_.get()}, 64, g.cchunk_begin.get(), g.cchunks,
                                                              part);
    lp_sum_kernel<<<grid_for((long long)g.K * 64), kT, 0, st_>>>(part, 64, g.clp_first.get(), g.K, g.inv_n.get(),
                                                                pooled_.get(), 128);
    PB_CUDA_CHECK(cudaGetLastError());
    if (g.m > 0) {
        chunk_kernel<<<std::min(g.rchunks, 148 * 8), 64, 0, st_>>>(PoolF{hc3_.get()}, 64, g.rchunk_begin.get(),
                                                                  g.rchunks, part);
        lp_sum_kernel<<<grid_for((long long)g.K * 64), kT, 0, st_>>>(part, 64, g.rlp_first.get(), g.K, g.inv_m.get(),
                                                                    pooled_.get() + 64, 128);
    } else {
        PB_CUDA_CHECK(cudaMemset2DAsync(pooled_.get() + 64, 512, 0, 256, size_t(g.K), st_));
    }
    rho_kernel<<<grid_for((long long)g.K * 32), kT, 0, st_>>>(pooled_.get(), g.K, pr + GnnParams::kHeadW, rho_.get());
    PB_CUDA_CHECK(cudaGetLastError());
}

double GnnModel::backward(const GnnGraph& g, bool grad) {
    if (last_ != &g) throw std::logic_error("GnnModel::backward: forward() was run on another graph");
    if (!g.has_targets) throw InvalidArgument("gnn: the graph has no targets");
    if (g.K == 0) return 0.0;
    const float* pr = pr_.get();
    float* part = part_.get();
    float* scratch = part_.get() + cap_chunks_ * kWide;
    float* G = g_.get();
    const float inv_k = 1.0f / float(g.K);
    float* drho = rho_.get() + cap_k_;
    // ---- loss per LP: x and y terms from chunk sums, omega term from rho ----
    std::vector<float> hl(size_t(3) * g.K);
    chunk_kernel<<<std::min(g.cchunks, 148 * 8), 32, 0, st_>>>(SqErrF{xhat_.get(), g.tx.get(), g.lp_col.get(),
                                                                      g.lw_x.get()},
                                                              1, g.cchunk_begin.get(), g.cchunks, part);
    lp_sum_kernel<<<grid_for(g.K), kT, 0, st_>>>(part, 1, g.clp_first.get(), g.K, nullptr, lp_sums_.get(), 1);
    if (g.m > 0) {
        chunk_kernel<<<std::min(g.rchunks, 148 * 8), 32, 0, st_>>>(
            SqErrF{yhat_.get(), g.ty.get(), g.lp_row.get(), g.lw_y.get()}, 1, g.rchunk_begin.get(), g.rchunks, part);
        lp_sum_kernel<<<grid_for(g.K), kT, 0, st_>>>(part, 1, g.rlp_first.get(), g.K, nullptr,
                                                    lp_sums_.get() + cap_k_, 1);
    } else {
        PB_CUDA_CHECK(cudaMemsetAsync(lp_sums_.get() + cap_k_, 0, size_t(g.K) * 4, st_));
    }
    PB_CUDA_CHECK(cudaGetLastError());
    std::vector<float> hrho(size_t(g.K)), htw(size_t(g.K));
    PB_CUDA_CHECK(cudaMemcpyAsync(hl.data(), lp_sums_.get(), size_t(g.K) * 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(hl.data() + g.K, lp_sums_.get() + cap_k_, size_t(g.K) * 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(hrho.data(), rho_.get(), size_t(g.K) * 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(htw.data(), g.tw.get(), size_t(g.K) * 4, cudaMemcpyDeviceToHost, st_));
    int hstatus = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&hstatus, status_.get(), 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (hstatus & kDevErrTimeout) throw DeviceTimeout("gnn: a tensor-core tile wait exceeded its time limit");
    double loss = 0.0;
    std::vector<float> hdrho(size_t(g.K));
    for (int k = 0; k < g.K; ++k) {
        const double dw = double(hrho[size_t(k)]) - double(htw[size_t(k)]);
        loss += double(hl[size_t(k)]) + double(hl[size_t(g.K + k)]) + dw * dw;
        hdrho[size_t(k)] = float(2.0 * dw) * inv_k;
    }
    loss /= g.K;
    if (!grad) return loss;

    // ---- heads ----
    PB_CUDA_CHECK(cudaMemsetAsync(G, 0, g_.bytes(), st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(drho, hdrho.data(), size_t(g.K) * 4, cudaMemcpyHostToDevice, st_));
    float* dxh = dagg_.get();                     // per-node head deltas (scratch)
    float* dyh = dagg_.get() + cap_n_;
    head_delta_kernel<<<grid_for(g.n), kT, 0, st_>>>(xhat_.get(), g.tx.get(), g.lp_col.get(), g.lw_x.get(), inv_k,
                                                    g.n, dxh);
    chunk_kernel<<<std::min(g.cchunks, 148 * 8), 96, 0, st_>>>(HeadGradF{hv3_.get(), dxh}, 65, g.cchunk_begin.get(),
                                                              g.cchunks, part);
    ordered_total(part, g.cchunks, 65, scratch, G + GnnParams::kHeadX, st_);
    if (g.m > 0) {
        head_delta_kernel<<<grid_for(g.m), kT, 0, st_>>>(yhat_.get(), g.ty.get(), g.lp_row.get(), g.lw_y.get(),
                                                        inv_k, g.m, dyh);
        chunk_kernel<<<std::min(g.rchunks, 148 * 8), 96, 0, st_>>>(HeadGradF{hc3_.get(), dyh}, 65,
                                                                  g.rchunk_begin.get(), g.rchunks, part);
        ordered_total(part, g.rchunks, 65, scratch, G + GnnParams::kHeadY, st_);
    }
    // w_w, b_w: sum_k drho_k [pooled_k ; 1]
    rho_grad_kernel<<<1, 160, 0, st_>>>(pooled_.get(), drho, g.K, G + GnnParams::kHeadW);
    PB_CUDA_CHECK(cudaGetLastError());
    head_back_kernel<<<grid_for((long long)g.n * 64), kT, 0, st_>>>(dxh, g.lp_col.get(), pr + GnnParams::kHeadX, drho,
                                                                   pr + GnnParams::kHeadW, g.inv_n.get(), g.n,
                                                                   dhv_.get());
    if (g.m > 0)
        head_back_kernel<<<grid_for((long long)g.m * 64), kT, 0, st_>>>(dyh, g.lp_row.get(), pr + GnnParams::kHeadY,
                                                                       drho, pr + GnnParams::kHeadW + 64,
                                                                       g.inv_m.get(), g.m, dhc_.get());
    PB_CUDA_CHECK(cudaGetLastError());

    // ---- message-passing layers, last to first ----
    const int wblocks_v = dense_blocks(dev_, g.n, 2), wblocks_c = dense_blocks(dev_, std::max(g.m, 1), 2);
    for (int l = kGnnLayers - 1; l >= 0; --l) {
        const bf16* out_c = l + 1 < kGnnLayers ? xc_[l + 1].get() : hc3_.get();
        const bf16* out_v = l + 1 < kGnnLayers ? xv_[l + 1].get() : hv3_.get();
        const int ldo = l + 1 < kGnnLayers ? 128 : 64;
        // variable side
        dz_kernel<<<grid_for((long long)g.n * 64), kT, 0, st_>>>(dhv_.get(), out_v, ldo, g.n, dz_.get());
        chunk_kernel<<<std::min(g.cchunks, 148 * 8), 64, 0, st_>>>(BiasGradF{dz_.get()}, 64, g.cchunk_begin.get(),
                                                                  g.cchunks, part);
        ordered_total(part, g.cchunks, 64, scratch, G + GnnParams::layer_b(l, 1), st_);
        {
            const CUtensorMap mx = make_bf16_tile_map(xv_[l].get(), g.n, 128, 128, 128);
            const CUtensorMap mz = make_bf16_tile_map(dz_.get(), g.n, 64, 64, 128);
            dense_dw_kernel<<<wblocks_v, kDenseThreads, DwSmem::kBytes, st_>>>(mx, mz, wpart_.get(), g.n, status_.get());
            PB_CUDA_CHECK(cudaGetLastError());
            dw_reduce_kernel<<<grid_for(64 * 128), kT, 0, st_>>>(wpart_.get(), wblocks_v, G + GnnParams::layer_w(l, 1));
            const CUtensorMap mwt = make_bf16_tile_map(wt_.get() + size_t(2 * l + 1) * 64 * 128, 128, 64, 64, 128);
            dense_dx_kernel<<<dense_blocks(dev_, g.n, 4), kDenseThreads, DxSmem::kBytes, st_>>>(
                mz, mwt, dhv_.get(), dagg_.get(), g.n, status_.get());
            PB_CUDA_CHECK(cudaGetLastError());
        }
        if (g.m > 0) {
            // agg_v backward: dh_c[i] += sum_j A_ij/(s_a deg_j) dagg_v[j]
            aggregate_bwd_kernel<<<grid_for((long long)g.m * 32), kT, 0, st_>>>(g.rp.get(), g.ci.get(),
                                                                                g.coef_c.get(), dagg_.get(),
                                                                                dhc_.get(), g.m);
            // constraint side
            dz_kernel<<<grid_for((long long)g.m * 64), kT, 0, st_>>>(dhc_.get(), out_c, ldo, g.m, dz_.get());
            chunk_kernel<<<std::min(g.rchunks, 148 * 8), 64, 0, st_>>>(BiasGradF{dz_.get()}, 64,
                                                                      g.rchunk_begin.get(), g.rchunks, part);
            ordered_total(part, g.rchunks, 64, scratch, G + GnnParams::layer_b(l, 0), st_);
            const CUtensorMap mx = make_bf16_tile_map(xc_[l].get(), g.m, 128, 128, 128);
            const CUtensorMap mz = make_bf16_tile_map(dz_.get(), g.m, 64, 64, 128);
            dense_dw_kernel<<<wblocks_c, kDenseThreads, DwSmem::kBytes, st_>>>(mx, mz, wpart_.get(), g.m, status_.get());
            PB_CUDA_CHECK(cudaGetLastError());
            dw_reduce_kernel<<<grid_for(64 * 128), kT, 0, st_>>>(wpart_.get(), wblocks_c, G + GnnParams::layer_w(l, 0));
            const CUtensorMap mwt = make_bf16_tile_map(wt_.get() + size_t(2 * l) * 64 * 128, 128, 64, 64, 128);
            dense_dx_kernel<<<dense_blocks(dev_, g.m, 4), kDenseThreads, DxSmem::kBytes, st_>>>(
                mz, mwt, dhc_.get(), dagg_.get(), g.m, status_.get());
            PB_CUDA_CHECK(cudaGetLastError());
            // agg_c backward: dh_v[j] += sum_i A_ij/(s_a deg_i) dagg_c[i]
            aggregate_bwd_kernel<<<grid_for((long long)g.n * 32), kT, 0, st_>>>(g.tp.get(), g.ti.get(),
                                                                                g.tcoef_r.get(), dagg_.get(),
                                                                                dhv_.get(), g.n);
            PB_CUDA_CHECK(cudaGetLastError());
        }
    }
    // ---- input layers ----
    inlayer_grad_kernel<<<std::min(g.cchunks, 148 * 16), 64, 0, st_>>>(dhv_.get(), xv_[0].get(), 128, g.fv.get(),
                                                                         g.cchunk_begin.get(), g.cchunks, part);
    ordered_total(part, g.cchunks, kWide, scratch, G + GnnParams::kVinW, st_);
    if (g.m > 0) {
        inlayer_grad_kernel<<<std::min(g.rchunks, 148 * 16), 64, 0, st_>>>(dhc_.get(), xc_[0].get(), 128, g.fc.get(),
                                                                           g.rchunk_begin.get(), g.rchunks, part);
        ordered_total(part, g.rchunks, kWide, scratch, G + GnnParams::kCinW, st_);
    }
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaMemcpyAsync(&hstatus, status_.get(), 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (hstatus & kDevErrTimeout) throw DeviceTimeout("gnn: a tensor-core tile wait exceeded its time limit");
    return loss;
}

void GnnModel::adam_step(float lr) {
    ++adam_t_;
    const float c1 = float(1.0 / (1.0 - std::pow(0.9, double(adam_t_))));
    const float c2 = float(1.0 / (1.0 - std::pow(0.999, double(adam_t_))));
    adam_kernel<<<grid_for(GnnParams::kCount), kT, 0, st_>>>(p_.get(), g_.get(), am_.get(), av_.get(),
                                                            GnnParams::kCount, lr, c1, c2);
    PB_CUDA_CHECK(cudaGetLastError());
    refresh_weights();
}

void GnnModel::predict(const GnnGraph& g, double* const* x, double* const* y, double* omega) {
    if (last_ != &g) throw std::logic_error("GnnModel::predict: forward() was run on another graph");
    if (g.K == 0) return;
    std::vector<float> hx(size_t(g.n)), hy(size_t(g.m)), hr(size_t(g.K));
    PB_CUDA_CHECK(cudaMemcpyAsync(hx.data(), xhat_.get(), size_t(g.n) * 4, cudaMemcpyDeviceToHost, st_));
    if (g.m) PB_CUDA_CHECK(cudaMemcpyAsync(hy.data(), yhat_.get(), size_t(g.m) * 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaMemcpyAsync(hr.data(), rho_.get(), size_t(g.K) * 4, cudaMemcpyDeviceToHost, st_));
    int hstatus = 0;
    PB_CUDA_CHECK(cudaMemcpyAsync(&hstatus, status_.get(), 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
    if (hstatus & kDevErrTimeout) throw DeviceTimeout("gnn: a tensor-core tile wait exceeded its time limit");
    for (int q = 0; q < g.K; ++q) {
        const int k = g.index[size_t(q)];
        const double sa = g.s_a[size_t(q)], sb = g.s_b[size_t(q)], sc = g.s_c[size_t(q)];
        if (x && x[k]) {
            for (int j = g.c0[size_t(q)]; j < g.c0[size_t(q) + 1]; ++j) {
                double v = double(hx[size_t(j)]) * sb / sa;
                if (g.h_vhi[size_t(j)] < 1e29 && v > g.h_vhi[size_t(j)]) v = g.h_vhi[size_t(j)];
                if (g.h_vlo[size_t(j)] > -1e29 && v < g.h_vlo[size_t(j)]) v = g.h_vlo[size_t(j)];
                x[k][j - g.c0[size_t(q)]] = v;
            }
        }
        if (y && y[k])
            for (int i = g.r0[size_t(q)]; i < g.r0[size_t(q) + 1]; ++i)
                y[k][i - g.r0[size_t(q)]] = double(hy[size_t(i)]) * sc / sa;
        if (omega) {
            const double rho = std::min(10.0, std::max(-10.0, double(hr[size_t(q)])));
            omega[k] = g.omega_ref[size_t(q)] * std::exp(rho);
        }
    }
}

size_t GnnModel::trace_size(const GnnGraph& g) const {
    return size_t(kGnnLayers) * (size_t(g.m) + size_t(g.n)) * 128 + (size_t(g.m) + size_t(g.n)) * 64 + size_t(g.n) +
           size_t(g.m) + size_t(g.K) * 129;
}

namespace {
__global__ void bf16_to_f32_kernel(const bf16* __restrict__ src, long long count, float* __restrict__ dst) {
    GNN_STRIDE(i, count) dst[i] = bf(src[i]);
}
}  // namespace

void GnnModel::trace(const GnnGraph& g, float* host) const {
    if (last_ != &g) throw std::logic_error("GnnModel::trace: forward() was run on another graph");
    const size_t total = trace_size(g);
    if (total == 0) return;
    DevBuf<float> t(total);
    size_t off = 0;
    auto conv = [&](const bf16* src, size_t count) {
        if (count) bf16_to_f32_kernel<<<grid_for((long long)count), kT, 0, st_>>>(src, (long long)count, t.get() + off);
        off += count;
    };
    auto copy = [&](const float* src, size_t count) {
        if (count)
            PB_CUDA_CHECK(cudaMemcpyAsync(t.get() + off, src, count * 4, cudaMemcpyDeviceToDevice, st_));
        off += count;
    };
    for (int l = 0; l < kGnnLayers; ++l) conv(xc_[l].get(), size_t(g.m) * 128);
    for (int l = 0; l < kGnnLayers; ++l) conv(xv_[l].get(), size_t(g.n) * 128);
    conv(hc3_.get(), size_t(g.m) * 64);
    conv(hv3_.get(), size_t(g.n) * 64);
    copy(xhat_.get(), size_t(g.n));
    copy(yhat_.get(), size_t(g.m));
    copy(pooled_.get(), size_t(g.K) * 128);
    copy(rho_.get(), size_t(g.K));
    PB_CUDA_CHECK(cudaGetLastError());
    PB_CUDA_CHECK(cudaMemcpyAsync(host, t.get(), total * 4, cudaMemcpyDeviceToHost, st_));
    PB_CUDA_CHECK(cudaStreamSynchronize(st_));
}

}  // namespace pb
