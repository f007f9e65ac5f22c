// ceiling.cu — the device's random-gather ceiling, measured.
//
// On an LP whose column indices are uniform random, every non-zero of a
// product costs one 4-byte gather from a random L2 sector, and what bounds the
// product is the rate at which the GPU serves such gathers, not HBM
// bandwidth.  This kernel issues nothing but those gathers: each thread loads
// kGathers entries of x at hashed uniform indices (no index array is read, so
// no other traffic competes), 16 loads in flight per thread, a persistent grid
// of 8 blocks per SM.  The benchmark reports each product's gathers per
// second as a fraction of this rate, beside its HBM fraction.
#include <algorithm>
#include <vector>

#include "common.cuh"

namespace pb {
namespace {

constexpr int kCeilThreads = 256;
constexpr int kCeilBlocksPerSm = 8;
constexpr int kGathers = 256;   // per thread, a multiple of 16

// Written only when a thread's sum hits one exact value, so the compiler must
// keep every load; the value itself is never used.
__device__ float g_ceiling_sink;

__device__ __forceinline__ uint32_t mix32(uint32_t a) {
    a ^= a >> 16; a *= 0x7feb352dU; a ^= a >> 15; a *= 0x846ca68bU; a ^= a >> 16;
    return a;
}

// cached: ld.global.ca (L1-cached) instead of ld.global.cg.  Every index is
// __umulhi(h, n) < n.
template <bool kCached>
__global__ void __launch_bounds__(kCeilThreads)
    gather_ceiling_kernel(const float* __restrict__ x, uint32_t n) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    float acc = 0.f;
    for (int k0 = 0; k0 < kGathers; k0 += 16) {
        float v[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const uint32_t h = mix32(tid * 0x9E3779B9u + uint32_t(k0 + j) * 0x85ebca6bu + 0x1234567u);
            const uint32_t idx = __umulhi(h, n);
            v[j] = kCached ? __ldca(x + idx) : __ldcg(x + idx);
        }
#pragma unroll
        for (int j = 0; j < 16; ++j) acc += v[j];
    }
    if (acc == 12345.678f) g_ceiling_sink = acc;
}

}  // namespace

// Median over `reps` timed launches of the gathers per second from x[0, n).
double measure_gather_rate(const float* d_x, int n, bool cached, int reps) {
    if (n <= 0 || !d_x) throw InvalidArgument("gather ceiling: x must be a device array with n > 0");
    if (reps < 1) reps = 1;
    int dev = 0, sms = 0;
    PB_CUDA_CHECK(cudaGetDevice(&dev));
    PB_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int grid = kCeilBlocksPerSm * sms;
    cudaStream_t st = nullptr;
    PB_CUDA_CHECK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<float> ms(static_cast<size_t>(reps));
    try {
        PB_CUDA_CHECK(cudaEventCreate(&e0));
        PB_CUDA_CHECK(cudaEventCreate(&e1));
        auto launch = [&] {
            if (cached) gather_ceiling_kernel<true><<<grid, kCeilThreads, 0, st>>>(d_x, uint32_t(n));
            else gather_ceiling_kernel<false><<<grid, kCeilThreads, 0, st>>>(d_x, uint32_t(n));
            PB_CUDA_CHECK(cudaGetLastError());
        };
        launch();   // warm-up: x into L2
        for (int r = 0; r < reps; ++r) {
            PB_CUDA_CHECK(cudaEventRecord(e0, st));
            launch();
            PB_CUDA_CHECK(cudaEventRecord(e1, st));
            PB_CUDA_CHECK(cudaEventSynchronize(e1));
            PB_CUDA_CHECK(cudaEventElapsedTime(&ms[size_t(r)], e0, e1));
        }
    } catch (...) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaStreamDestroy(st);
        throw;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    PB_CUDA_CHECK(cudaStreamDestroy(st));
    std::sort(ms.begin(), ms.end());
    const double med = ms[ms.size() / 2];
    const double gathers = double(grid) * kCeilThreads * kGathers;
    return gathers / (med * 1e-3);
}

}  // namespace pb
