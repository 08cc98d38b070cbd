// umma.cuh — fifth-generation tensor-core primitives for sm_100a (inline PTX):
// tensor-memory allocation, tcgen05.mma with shared-memory operand
// descriptors, commit to an mbarrier, tensor-memory loads, and the fences
// that order them against thread synchronisation.
//
// Operand layout used with these helpers: K-major, no swizzle.  An R x K
// bf16 matrix (R = M rows of A or N rows of B) is stored as 8 x 8 "core
// matrices" of 128 contiguous bytes (8 rows of 16 B); element (r, k) lives at
//   (r / 8) * SBO + (k / 8) * LBO + (r % 8) * 16 + (k % 8) * 2
// with LBO = 128 (core matrices adjacent along K) and SBO = K / 8 * 128 (the
// next 8 rows).  One MMA consumes K = 16, i.e. two core matrices along K, so
// k-step s starts 256 * s bytes into the operand.
#pragma once

#include <cstdint>

namespace srt {

constexpr uint32_t ERR_MMA_TIMEOUT = 0x8u;

__device__ __forceinline__ uint32_t smem_u32addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Byte offset of element (r, k) in the K-major core-matrix layout of a matrix with K columns.
__host__ __device__ constexpr uint32_t umma_offset(uint32_t r, uint32_t k, uint32_t K) {
    return (r / 8u) * (K / 8u * 128u) + (k / 8u) * 128u + (r % 8u) * 16u + (k % 8u) * 2u;
}

// Shared-memory matrix descriptor (tcgen05): start address >> 4 in bits
// 0..13, leading-dimension byte offset >> 4 in 16..29, stride-dimension byte
// offset >> 4 in 32..45, descriptor version 1 in 46..47, base offset 0, no
// swizzle (layout type 0 in bits 61..63).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4..5 = 1), BF16
// A and B (bits 7..9 = 1, 10..12 = 1), both K-major, N >> 3 in bits 17..22,
// M >> 4 in bits 24..28.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// Tensor-memory allocation: one full warp; the base address is written to *dst.
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32addr(dst)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n"
        "}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// The mbarrier completes one arrival when every tcgen05.mma issued so far by
// this thread has finished.
__device__ __forceinline__ void umma_commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32addr(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32addr(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32addr(mbar)), "r"(parity)
        : "memory");
    return ok != 0u;
}
// Bounded wait: false after `limit` polls (the caller records the timeout).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(mbar, parity)) return true;
    return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
// Shared-memory writes of the threads become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp w reads
// lanes 32 w .. 32 w + 31; taddr carries the lane in bits 16..31).  The
// registers are valid only after tmem_wait16 on the same array, which takes
// them as operands so that no use can move above the wait.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait16(uint32_t (&r)[16]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;\n"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])
                 :
                 : "memory");
}

}  // namespace srt
