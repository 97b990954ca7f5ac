// learned.cuh -- the learned warm start inside the transport step.
//
// The step's Newton solves produce, every step, (component totals ->
// log10 free components) pairs.  With learning on (CL_OPT_EQ_LEARN), the
// one-launch step stores a sampled subset of its converged pairs in a ring
// on the device; every `interval` steps the library trains its network
// (n_comp -> 64 -> 64 -> n_comp, GELU; the trainer of speciation.cu, BF16
// tensor-core forward/backward with FP32 master weights) on the ring, and
// from then on a voxel with no previous solution of its own (the first step,
// a reopened or newly stored voxel, after a reset) starts Newton from the
// network's guess where that guess has a smaller relative mass-balance
// residual than the reference's cold start, falling back to the cold start
// after warm_iter iterations.  Newton's 1e-10 relative residual still decides convergence,
// so the fields do not depend on the guess beyond that tolerance.
#pragma once
#include <cmath>

namespace cl {

constexpr int kLearnHidden = 64;

__device__ __forceinline__ float learn_gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }

// the network's start x from the totals T, with the FP32 master weights
// (layout W1[H][NC] b1[H] W2[H][H] b2[H] W3[NC][H] b3[NC]) and the
// standardisation norm = mu_in[NC] sd_in[NC] mu_out[NC] sd_out[NC] of the
// trainer (inputs log10 T, outputs x - log10 T)
// values in and out by value: a call with pointers would put the caller's
// arrays on the stack for the whole reaction chain
template <int NC>
struct LearnVec {
    double v[NC];
};

template <int NC>
__device__ __noinline__ LearnVec<NC> learn_start(const float* __restrict__ w, const float* __restrict__ norm,
                                                 const LearnVec<NC> Tv) {
    const double* T = Tv.v;
    LearnVec<NC> out;
    double* x = out.v;
    constexpr int H = kLearnHidden;
    const float* W1 = w;
    const float* b1 = W1 + H * NC;
    const float* W2 = b1 + H;
    const float* b2 = W2 + H * H;
    const float* W3 = b2 + H;
    const float* b3 = W3 + NC * H;
    float u[NC], xin[NC], y[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        u[k] = (float)log10(fmax(T[k], 1e-30));
        xin[k] = (u[k] - __ldg(norm + k)) / __ldg(norm + NC + k);
        y[k] = __ldg(b3 + k);
    }
    float h1[H];
#pragma unroll
    for (int o = 0; o < H; ++o) {
        float z = __ldg(b1 + o);
#pragma unroll
        for (int k = 0; k < NC; ++k) z = fmaf(__ldg(W1 + o * NC + k), xin[k], z);
        h1[o] = learn_gelu(z);
    }
    for (int o = 0; o < H; ++o) {
        float z = __ldg(b2 + o);
#pragma unroll 16
        for (int i = 0; i < H; ++i) z = fmaf(__ldg(W2 + o * H + i), h1[i], z);
        const float a = learn_gelu(z);
#pragma unroll
        for (int k = 0; k < NC; ++k) y[k] = fmaf(__ldg(W3 + k * H + o), a, y[k]);
    }
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        const double v = (double)u[k] + (double)__ldg(norm + 2 * NC + k) + (double)__ldg(norm + 3 * NC + k) * (double)y[k];
        x[k] = fmin(fmax(v, -30.0), 1.0);
    }
    return out;
}

// the pair of a converged voxel goes to the ring when its site hash falls in
// this step's sample (one voxel in 2^shift)
__device__ __forceinline__ bool learn_sampled(uint32_t n, uint32_t salt, uint32_t mask) {
    uint32_t h = n * 0x9E3779B1u ^ salt;
    h ^= h >> 16; h *= 0x85EBCA6Bu; h ^= h >> 13;
    return (h & mask) == 0;
}

template <int NC>
__device__ __forceinline__ void learn_store(double* pT, double* pX, unsigned long long* count, int64_t cap,
                                            const double* T, const double* x) {
    const unsigned long long i = atomicAdd(count, 1ull);
    if ((int64_t)i >= cap) return;
#pragma unroll
    for (int k = 0; k < NC; ++k) { pT[i * NC + k] = T[k]; pX[i * NC + k] = x[k]; }
}

}  // namespace cl
