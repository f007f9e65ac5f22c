// common.cuh — error plumbing, status codes and sm_100a PTX helpers shared by
// every translation unit of libpramaan_b200.
//
// Error convention (mirrors src/gpu/cuda_utils.cuh:8-15 of the reference):
// a failing CUDA call raises std::runtime_error("CUDA error in <file>:<line> -
// <msg>").  The extern "C" layer catches it, stores the text in a
// thread-local buffer (pramaan_last_error) and returns a negative status.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <mutex>
#include <shared_mutex>
#include <stdexcept>
#include <string>

#include "../../include/pramaan_b200.h"

#define PB_CUDA_CHECK(call)                                                              \
    do {                                                                                 \
        cudaError_t pb_err__ = (call);                                                   \
        if (pb_err__ != cudaSuccess) {                                                   \
            throw ::pb::CudaError(std::string("CUDA error in ") + __FILE__ + ":" +       \
                                  std::to_string(__LINE__) + " - " +                     \
                                  cudaGetErrorString(pb_err__));                         \
        }                                                                                \
    } while (0)

namespace pb {

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct InvalidArgument : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};
// A device-side bounded wait gave up (see kErrTimeout in the device status word).
struct DeviceTimeout : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Graph captures run in thread-local mode, which still breaks when another
// host thread makes a call that synchronises with every stream of the device
// (cudaDeviceSynchronize, cudaFree, cudaFreeHost, cudaMallocHost) while the
// capture is open.  Each capture holds this gate shared from begin to end and
// each such call holds it exclusively, so solves running concurrently from
// several host threads stay legal.
inline std::shared_mutex& capture_gate() {
    static std::shared_mutex m;
    return m;
}
inline bool& capture_open_here() {
    thread_local bool open = false;
    return open;
}
struct CaptureScope {
    std::shared_lock<std::shared_mutex> lk{capture_gate()};
    CaptureScope() { capture_open_here() = true; }
    ~CaptureScope() { capture_open_here() = false; }
};
// A thread whose own capture is open never takes the gate exclusively (it
// would wait on itself); CUDA rejects the call in that thread instead.
struct DeviceSyncScope {
    std::unique_lock<std::shared_mutex> lk;
    DeviceSyncScope() {
        if (!capture_open_here()) lk = std::unique_lock<std::shared_mutex>(capture_gate());
    }
};
template <class T>
cudaError_t pinned_alloc(T** p, size_t bytes) {
    DeviceSyncScope gate;
    return cudaMallocHost(reinterpret_cast<void**>(p), bytes);
}

// Device status word bits (written by kernels, read by the host after a sync).
enum : int {
    kDevOk = 0,
    kDevErrTimeout = 1,      // an mbarrier wait on a TMA bulk copy exceeded its time limit
    kDevErrNonFinite = 2,    // a NaN/Inf appeared in an iterate
};

// Wait limit for every spin on an mbarrier (nanoseconds of %globaltimer).
constexpr unsigned long long kWaitLimitNs = 1000000000ull;   // 1 s

// ---------------------------------------------------------------------------
// Device helpers (inline PTX, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_timer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Makes initialised mbarriers visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive on `bar` (count 1) and add `bytes` to its expected transaction count.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: returns false when the phase did not complete within
// kWaitLimitNs.  Never spins forever.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_timer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_timer_ns() - t0 > kWaitLimitNs) return false;
    }
}

// try_wait with a suspend-time hint: a thread whose phase has not completed
// sleeps in hardware for up to `hint_ns` instead of returning at once, so
// waiting warps do not take issue slots from the warps that have work.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Bounded wait that sleeps between checks (see mbar_try_wait_sleep); gives
// up after kWaitLimitNs like mbar_wait_bounded.
__device__ __forceinline__ bool mbar_wait_bounded_sleep(uint64_t* bar, uint32_t parity) {
    constexpr uint32_t kHintNs = 20000;
    if (mbar_try_wait_sleep(bar, parity, kHintNs)) return true;
    const unsigned long long t0 = global_timer_ns();
    while (true) {
        if (mbar_try_wait_sleep(bar, parity, kHintNs)) return true;
        if (global_timer_ns() - t0 > kWaitLimitNs) return false;
    }
}

// Programmatic dependent launch.  A kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may start while the
// previous kernel of its stream is still running; grid_dep_wait() blocks
// until that kernel has completed and its memory is visible, so everything
// before it may only read data no kernel writes (tile records, constants).
// grid_dep_launch() lets the next such kernel be scheduled early.  Both are
// no-ops for kernels launched without the attribute.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// L2 eviction-priority policy for streamed (read-once) data.
// L2 eviction-priority policy for data read again by the next launch (an
// operand that fits in L2 with its vectors).
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// 1-D TMA bulk copy global -> shared, completing on `bar` (complete_tx).
// Both addresses must be 16-byte aligned and `bytes` a multiple of 16.
__device__ __forceinline__ void tma_bulk_g2s(void* smem_dst, const void* gsrc, unsigned bytes,
                                             uint64_t* bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// Bulk prefetch of [gsrc, gsrc + bytes) into L2 (no shared memory, no
// completion to wait for).  16-byte aligned address, size a multiple of 16.
__device__ __forceinline__ void bulk_prefetch_l2(const void* gsrc, unsigned bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gsrc), "r"(bytes) : "memory");
}

template <typename T>
__device__ __forceinline__ T ld_cg(const T* p) {
    return __ldcg(p);
}

// Atomic max for non-negative doubles: the IEEE bit patterns of non-negative
// doubles order like unsigned integers, so an integer max is exact and
// independent of arrival order.
__device__ __forceinline__ void atomic_max_nonneg(double* addr, double v) {
    if (!(v > 0.0)) return;   // also drops NaN (recorded separately)
    atomicMax(reinterpret_cast<unsigned long long*>(addr),
              static_cast<unsigned long long>(__double_as_longlong(v)));
}

inline int ceil_div(long long a, long long b) { return static_cast<int>((a + b - 1) / b); }

}  // namespace pb
