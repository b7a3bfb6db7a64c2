// Fifth-generation tensor-core (tcgen05) helpers for sm_100a, in inline PTX.
//
// Used by the split-precision form of the azimuth transforms: small dense DFT tiles run as
// bf16 x bf16 -> fp32 matrix products, A (data) in tensor memory (TMEM), B (DFT matrix) in
// shared memory in the canonical no-swizzle K-major layout, the accumulator D in TMEM.  One
// thread issues the products; completion is signalled through tcgen05.commit to a
// shared-memory mbarrier whose waits are bounded (tma.cuh).
//
// Shared-memory operand layout (no swizzle, K-major, 16-bit elements): a "core matrix" is
// 8 rows x 8 elements (16 bytes per row, 128 contiguous bytes).  Element (row, k) of an
// operand with K elements per row lies at byte
//     (row / 8) * SBO + (k / 8) * LBO + (row % 8) * 16 + (k % 8) * 2
// with LBO = 128 (K-adjacent core matrices) and SBO = 128 * K / 8 (row-adjacent groups)
// (umma_offset in params.h).  One kind::f16 product consumes K = 16, i.e. two core-matrix
// columns; the descriptor of k-step s starts 2 * s * LBO bytes further.  In TMEM, row i of A
// is lane i and K elements 2j, 2j + 1 share 32-bit column j (the lower index in the low half).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "params.h"
#include "tma.cuh"

namespace asarf {

constexpr unsigned kErrMmaTimeout = 1u << 5;

// Shared-memory matrix descriptor: start address, leading / stride byte offsets (>> 4),
// descriptor version 1 (bits 46-47), no swizzle (bits 61-63 = 0).
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= static_cast<uint64_t>((saddr >> 4) & 0x3FFFu);
    d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
    d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
    d |= static_cast<uint64_t>(1) << 46;
    return d;
}

// Instruction descriptor of kind::f16: D fp32, A and B bf16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
    return (1u << 4)                                   // D format f32
           | (1u << 7)                                 // A format bf16
           | (1u << 10)                                // B format bf16
           | (static_cast<uint32_t>(n >> 3) << 17)     // N / 8
           | (static_cast<uint32_t>(m >> 4) << 24);    // M / 16
}

// TMEM allocation by one whole warp; the base address is written to *dst (shared memory).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[taddr] (+)= A * B with A in TMEM (lanes = rows, two 16-bit K elements per 32-bit column,
// the lower K index in the low half) and B in shared memory, one elected thread.
__device__ __forceinline__ void umma_bf16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                             bool accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.u32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
        : "memory");
}

// 8 consecutive 32-bit TMEM columns of this thread's lane from registers (warp w writes lanes
// 32 (w % 4) ..); tmem_wait_st makes the stores complete before a barrier.
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* v) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
                 : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Arrive once on `bar` when every product issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane (warp w reads lanes 32 (w % 4) ..).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    // the wait names the loaded registers, so nothing that reads them is scheduled before it
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// bf16 hi + lo split of two floats, packed (low half = first value): hi = bf16(x),
// lo = bf16(x - hi); x - hi is exact in fp32, so hi + lo carries 16 significant bits.
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
    uint32_t h;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(h) : "f"(b), "f"(a));
    const float ha = __uint_as_float(h << 16);
    const float hb = __uint_as_float(h & 0xFFFF0000u);
    uint32_t l;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(l) : "f"(b - hb), "f"(a - ha));
    hi = h;
    lo = l;
}

}  // namespace asarf
