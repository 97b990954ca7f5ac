// umma.cuh -- the fifth-generation tensor core (tcgen05) for one CTA:
// accumulators in tensor memory (TMEM), operands in shared memory described
// by 64-bit matrix descriptors, completion through an mbarrier.
//
// Operand layout (both operands K-major, no swizzle): a tile of R rows by K
// BF16 elements is stored as 8x8 core matrices of 128 contiguous bytes (row r
// of a core matrix at byte 16 r); core matrix (row group g, K chunk c) starts
// at byte (g * K/8 + c) * 128.  One MMA of K = 16 reads two K chunks, so its
// descriptor has the leading-dimension byte offset 128 (the next K chunk) and
// the stride-dimension byte offset K/8 * 128 (the next group of 8 rows).
//
// The MMA computes D[m][n] (+)= sum_k A[m][k] B[n][k] with M = 128 rows in
// TMEM lanes 0..127 and N FP32 columns; a warp w of the CTA reads lanes
// 32 w .. 32 w + 31 (tcgen05.ld shape 32x32b), so thread t of warp w holds
// row 32 w + t.
//
// The bit layouts of the descriptors follow the sm100 UMMA definitions
// (matrix descriptor: start address >> 4 in bits 0-13, leading byte offset
// >> 4 in 16-29, stride byte offset >> 4 in 32-45, version 1 in 46-47,
// layout type in 61-63; instruction descriptor for kind::f16: D format in
// bits 4-5, A and B formats in 7-9 and 10-12, transposes in 15 and 16,
// N >> 3 in 17-22, M >> 4 in 24-28).
#pragma once
#include <cstdint>

namespace cl {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (row, k) of a K-major tile with kch = K / 8 chunks
__device__ __forceinline__ uint32_t umma_off(int row, int k, int kch) {
    return (uint32_t)((((row >> 3) * kch + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

// descriptor of the K = 16 slice kb of a K-major tile at shared address base
__device__ __forceinline__ uint64_t umma_desc(uint32_t base, int kb, int kch) {
    const uint32_t start = base + (uint32_t)(kb * 256);
    const uint64_t lbo = 128u >> 4, sbo = (uint64_t)(kch * 128) >> 4;
    return (uint64_t)((start >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// kind::f16 with BF16 A and B, FP32 D, both K-major, M = 128
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// one MMA issued by the calling thread; accumulate selects D += A B over D = A B
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
        :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(z) : "memory");
}

// the mbarrier at bar completes a phase when the calling thread's earlier MMAs are done
__device__ __forceinline__ void umma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(bar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// waits for the phase of the given parity to complete; false after `limit`
// polls (the caller reports an error instead of waiting for ever)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done) : "r"(bar), "r"(parity) : "memory");
        if (done) return true;
    }
    return false;
}

// generic-proxy writes to shared memory made visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM allocation by one whole warp; the base address lands in *dst (shared)
__device__ __forceinline__ void tmem_alloc(uint32_t dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(dst), "r"(ncols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(base), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's lane, starting at taddr
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace cl
