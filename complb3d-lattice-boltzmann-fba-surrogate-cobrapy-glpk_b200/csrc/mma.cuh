// mma.cuh -- warp-level BF16 tensor-core tiles (FP32 accumulate) for the
// small networks: the learned speciation warm start and the surrogate rate
// network.  Operands live in shared memory: A row-major [m][k] and B given as
// its transpose BT row-major [n][k], so that every fragment element pair is
// one aligned 32-bit load.  Row pitches are chosen with (pitch/2) % 32 == 4 or
// 12 so the eight rows a fragment touches land in distinct banks.
#pragma once
#include <cuda_bf16.h>
#include <cstdint>

namespace cl {

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16* p) {
    return *reinterpret_cast<const uint32_t*>(p);
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t*>(&v);
}

// D = A(16x16, row) * B(16x8, col) + C, bf16 inputs, f32 accumulate
__device__ __forceinline__ void mma_bf16_16816(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
        "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// acc(16x8 tile at rows m0.., cols n0..) += A[m0:m0+16, 0:K] * BT[n0:n0+8, 0:K]^T
// acc layout: acc[0..1] = (m0+g, n0+2t..+1), acc[2..3] = (m0+g+8, n0+2t..+1)
__device__ __forceinline__ void warp_tile(float* acc, const __nv_bfloat16* A, int lda, int m0,
                                          const __nv_bfloat16* BT, int ldb, int n0, int K) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const __nv_bfloat16* a_lo = A + (m0 + g) * lda + 2 * t;
    const __nv_bfloat16* a_hi = A + (m0 + g + 8) * lda + 2 * t;
    const __nv_bfloat16* b = BT + (n0 + g) * ldb + 2 * t;
    for (int k = 0; k < K; k += 16) {
        mma_bf16_16816(acc, ld32(a_lo + k), ld32(a_hi + k), ld32(a_lo + k + 8), ld32(a_hi + k + 8),
                       ld32(b + k), ld32(b + k + 8));
    }
}

}  // namespace cl
