// umma.cuh — sm_100a tensor-core plumbing for the dense layers of the
// warm-start network: 2-D TMA tile loads (cp.async.bulk.tensor), shared-memory
// matrix descriptors, tcgen05.mma (kind::f16, BF16 inputs, FP32 accumulator in
// tensor memory), tcgen05.commit and tcgen05.ld.
//
// Operand tiles are always loaded by TMA with the 128-byte swizzle from
// row-major BF16 arrays whose rows hold 64 (one box) or 128 (two boxes)
// elements, so every tile in shared memory is a stack of 1024-byte swizzle
// atoms (8 rows x 128 bytes).  Read along the row, a box is a K-major operand
// (K = the 64 elements of a row); read down the rows, the same box is an
// MN-major operand (K = the rows).  Descriptor fields follow the canonical
// layouts of the PTX ISA's tcgen05 "shared memory descriptor":
//   K-major,  SWIZZLE_128B: LBO = 16 B (unused), SBO = 1024 B between 8-row
//             groups; one K=16 step advances the start address by 32 B.
//   MN-major, SWIZZLE_128B: LBO = byte distance between 64-element MN chunks
//             (the second box), SBO = 1024 B between 8-row K groups; one K=16
//             step advances the start address by 2048 B.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "common.cuh"

namespace pb {
namespace umma {

// ---- descriptors -----------------------------------------------------------
constexpr uint32_t kSwizzle128B = 2;

__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= uint64_t((saddr & 0x3FFFFu) >> 4);              // start address, bits 0-13
    d |= uint64_t((lbo_bytes >> 4) & 0x3FFFu) << 16;      // leading byte offset, bits 16-29
    d |= uint64_t((sbo_bytes >> 4) & 0x3FFFu) << 32;      // stride byte offset, bits 32-45
    d |= uint64_t(1) << 46;                               // descriptor version (sm_100)
    d |= uint64_t(kSwizzle128B) << 61;                    // layout: 128-byte swizzle
    return d;
}

// Instruction descriptor of tcgen05.mma.kind::f16: BF16 A and B, FP32 D.
template <int M, int N, bool kAMajorMN, bool kBMajorMN>
__host__ __device__ constexpr uint32_t idesc_bf16() {
    static_assert(M == 128, "one CTA, M = 128");
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N in [16, 256], a multiple of 16");
    return (1u << 4)                       // D format: F32
           | (1u << 7)                     // A format: BF16
           | (1u << 10)                    // B format: BF16
           | (uint32_t(kAMajorMN) << 15)   // A major: 0 K, 1 MN
           | (uint32_t(kBMajorMN) << 16)   // B major
           | (uint32_t(N >> 3) << 17)      // N / 8
           | (uint32_t(M >> 4) << 24);     // M / 16
}

// ---- tensor memory ---------------------------------------------------------
// Executed by one whole warp; writes the allocated base address to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// ---- MMA -------------------------------------------------------------------
// D[tmem] (+)= A[smem] * B[smem]^T, issued by a single thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrives (once) on `bar` when every MMA issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// ---- tensor memory -> registers --------------------------------------------
// Warp w of the CTA reads lanes 32w..32w+31 (thread t: lane 32w+t), 32
// consecutive FP32 columns starting at `taddr`'s column.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
          "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
          "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
          "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ---- TMA -------------------------------------------------------------------
__device__ __forceinline__ void tma_prefetch_map(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}
// 2-D tiled load of the box at element coordinates (x, y) into shared memory;
// completes on `bar`.  x is always 0 or 64 here (a 16-byte multiple).
__device__ __forceinline__ void tma_load_2d(void* smem_dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace umma

// Host: a 2-D tensor map over a row-major BF16 array [rows][cols] (cols = 64
// or 128, row pitch `pitch_elems`), box = 64 columns x `box_rows` rows,
// 128-byte swizzle, out-of-range rows read as zero.
CUtensorMap make_bf16_tile_map(const void* base, long long rows, int cols, int pitch_elems, int box_rows);

}  // namespace pb
