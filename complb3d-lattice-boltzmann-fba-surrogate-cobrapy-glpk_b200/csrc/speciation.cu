// speciation.cu -- batched FP64 Newton speciation and its learned warm start.
//
// Batch solve: one voxel per thread.  A warm start (given or learned) gets at
// most warm_iter Newton iterations; voxels that have not converged by then are
// appended to a compact list and re-solved from the reference's cold start in
// a second launch, so a few slow voxels do not hold whole warps of fast ones.
//
// Learned warm start: an MLP n_comp -> 64 -> 64 -> n_comp with GELU hidden
// layers maps u = log10 T (standardised) to v = x - log10 T (standardised).
// Every contraction of the forward and backward passes is a BF16 tensor-core
// MMA with FP32 accumulation over 64-sample tiles staged in shared memory;
// master weights are FP32, the MMA operands BF16.  Training is plain Adam on
// the MSE of v, driven on the device by the library's own kernels on the pairs
// (T, x) that Newton produced.  Newton stays the arbiter: the network only picks
// the starting point.
#include "internal.h"
#include "newton.cuh"
#include "speciation_large.h"
#include "pcf.cuh"
#include "mma.cuh"
#include "umma.cuh"
#include <cmath>
#include <vector>
#include <random>
#include <algorithm>
#include <mutex>

namespace cl {

constexpr int H = CL_MLP_HIDDEN;   // 64
constexpr int TS = 64;             // samples per block tile
constexpr int KP = 16;             // padded input width
constexpr int NP = 16;             // padded output width (as a K dimension)
constexpr int P24 = 24, P72 = 72;  // row pitches (bf16 elements)
constexpr int MLP_THREADS = 128;

struct MlpDev {
    // BF16 operand copies, padded
    __nv_bfloat16* W1;   // [H][P24]  W1[h][k], k < nc
    __nv_bfloat16* W2;   // [H][P72]
    __nv_bfloat16* W2T;  // [H][P72]  W2T[i][o] = W2[o][i]
    __nv_bfloat16* W3;   // [8][P72]  W3[o][h], o < nc
    __nv_bfloat16* W3T;  // [H][P24]  W3T[h][o]
    float* b;            // b1[H] b2[H] b3[nc]
    float* norm;         // mu_in[nc] sd_in[nc] mu_out[nc] sd_out[nc]
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
    return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// shared-memory layout of one block (bytes)
struct MlpSmem {
    __nv_bfloat16 X[TS * P24], XT[KP * P72];
    __nv_bfloat16 W1[H * P24], W2[H * P72], W2T[H * P72], W3[8 * P72], W3T[H * P24];
    __nv_bfloat16 A1[TS * P72], A1T[H * P72], A2[TS * P72], A2T[H * P72];
    __nv_bfloat16 dY[TS * P24], dYT[NP * P72], dZ2[TS * P72], dZ2T[H * P72], dZ1T[H * P72];
    float D1[TS * H], D2[TS * H];
    float b[2 * H + 8];
    float db[2 * H + 8];
    float loss[MLP_THREADS];
};

// what the forward pass alone needs (inference): a quarter of MlpSmem, so
// several blocks share an SM
struct MlpSmemFwd {
    __nv_bfloat16 X[TS * P24];
    __nv_bfloat16 W1[H * P24], W2[H * P72], W3[8 * P72];
    __nv_bfloat16 A1[TS * P72], A2[TS * P72];
    float b[2 * H + 8];
};

template <class SM>
__device__ void load_weights(SM& s, const MlpDev& w, int nc) {
    auto cp = [](__nv_bfloat16* dst, const __nv_bfloat16* src, int n) {
        for (int i = threadIdx.x; i < n; i += blockDim.x) dst[i] = src[i];
    };
    cp(s.W1, w.W1, H * P24); cp(s.W2, w.W2, H * P72); cp(s.W3, w.W3, 8 * P72);
    if constexpr (sizeof(SM) == sizeof(MlpSmem)) { cp(s.W2T, w.W2T, H * P72); cp(s.W3T, w.W3T, H * P24); }
    for (int i = threadIdx.x; i < 2 * H + nc; i += blockDim.x) s.b[i] = w.b[i];
}

// Forward of one 64-sample tile whose standardised inputs are already in s.X
// (and s.XT when training).  Leaves A1/A2 (and transposes, D1/D2 when
// training) in shared memory; returns through y_out the standardised outputs
// of this thread's output fragments via callback.
template <bool TRAIN, class SM>
__device__ void mlp_forward_tile(SM& s, int nc, float (*yfrag)[4]) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // Z1 = X W1^T (64 x 64): 32 tiles, 8 per warp
    for (int q = 0; q < 8; ++q) {
        const int tile = warp * 8 + q, m0 = (tile >> 3) * 16, n0 = (tile & 7) * 8;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        warp_tile(acc, s.X, P24, m0, s.W1, P24, n0, KP);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int m = m0 + g + (r >> 1) * 8, n = n0 + 2 * t + (r & 1);
            const float z = acc[r] + s.b[n];
            const float a = gelu(z);
            s.A1[m * P72 + n] = __float2bfloat16_rn(a);
            if constexpr (TRAIN) { s.A1T[n * P72 + m] = __float2bfloat16_rn(a); s.D1[m * H + n] = gelu_d(z); }
        }
    }
    __syncthreads();
    // Z2 = A1 W2^T
    for (int q = 0; q < 8; ++q) {
        const int tile = warp * 8 + q, m0 = (tile >> 3) * 16, n0 = (tile & 7) * 8;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        warp_tile(acc, s.A1, P72, m0, s.W2, P72, n0, H);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int m = m0 + g + (r >> 1) * 8, n = n0 + 2 * t + (r & 1);
            const float z = acc[r] + s.b[H + n];
            const float a = gelu(z);
            s.A2[m * P72 + n] = __float2bfloat16_rn(a);
            if constexpr (TRAIN) { s.A2T[n * P72 + m] = __float2bfloat16_rn(a); s.D2[m * H + n] = gelu_d(z); }
        }
    }
    __syncthreads();
    // Y = A2 W3^T (64 x 8): one 16x8 tile per warp
    {
        const int m0 = warp * 16;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        warp_tile(acc, s.A2, P72, m0, s.W3, P72, 0, H);
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int n = 2 * t + (r & 1);
            yfrag[0][r] = (n < nc) ? acc[r] + s.b[2 * H + n] : 0.f;
        }
    }
}

// Gradient of the batch loss mean((y - target)^2) over `total` samples times
// nc outputs; each block adds its tiles' contributions and writes its partial
// sums in the oracle's parameter layout.
__global__ void __launch_bounds__(MLP_THREADS) mlp_grad_kernel(MlpDev w, int nc, const float* Xn, const float* Yn,
                                                               int64_t begin, int64_t count, float inv_scale,
                                                               float* part, int n_params) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmem& s = *reinterpret_cast<MlpSmem*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    load_weights(s, w, nc);
    for (int i = threadIdx.x; i < 2 * H + 8; i += blockDim.x) s.db[i] = 0.f;
    // zero the padded operand regions once
    for (int i = threadIdx.x; i < TS * P24; i += blockDim.x) { s.X[i] = __float2bfloat16_rn(0.f); s.dY[i] = __float2bfloat16_rn(0.f); }
    for (int i = threadIdx.x; i < KP * P72; i += blockDim.x) s.XT[i] = __float2bfloat16_rn(0.f);
    for (int i = threadIdx.x; i < NP * P72; i += blockDim.x) s.dYT[i] = __float2bfloat16_rn(0.f);
    float lsum = 0.f;
    float gW2[8][4], gW3[2][4], gW1[2][4];
#pragma unroll
    for (int q = 0; q < 8; ++q) for (int r = 0; r < 4; ++r) gW2[q][r] = 0.f;
#pragma unroll
    for (int q = 0; q < 2; ++q) for (int r = 0; r < 4; ++r) { gW3[q][r] = 0.f; gW1[q][r] = 0.f; }
    __syncthreads();
    const int64_t ntiles = (count + TS - 1) / TS;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t s0 = begin + tile * TS;
        const int valid = (int)min((int64_t)TS, begin + count - s0);
        for (int i = threadIdx.x; i < TS * nc; i += blockDim.x) {
            const int m = i / nc, k = i - m * nc;
            const float v = (m < valid) ? Xn[(s0 + m) * nc + k] : 0.f;
            s.X[m * P24 + k] = __float2bfloat16_rn(v);
            s.XT[k * P72 + m] = __float2bfloat16_rn(v);
        }
        __syncthreads();
        float yf[1][4];
        mlp_forward_tile<true>(s, nc, yf);
        // dY = inv_scale * 2 (y - target), zero for padded samples / outputs
        {
            const int m0 = warp * 16;
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + g + (r >> 1) * 8, n = 2 * t + (r & 1);
                float d = 0.f;
                if (n < nc && m < valid) {
                    const float e = yf[0][r] - Yn[(s0 + m) * nc + n];
                    lsum += e * e;
                    d = 2.f * e * inv_scale;
                }
                s.dY[m * P24 + n] = __float2bfloat16_rn(d);
                s.dYT[n * P72 + m] = __float2bfloat16_rn(d);
            }
        }
        __syncthreads();
        // dZ2 = (dY W3) * gelu'(Z2)   (64 x 64, K = 16)
        for (int q = 0; q < 8; ++q) {
            const int tl = warp * 8 + q, m0 = (tl >> 3) * 16, n0 = (tl & 7) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile(acc, s.dY, P24, m0, s.W3T, P24, n0, NP);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + g + (r >> 1) * 8, n = n0 + 2 * t + (r & 1);
                const float d = acc[r] * s.D2[m * H + n];
                s.dZ2[m * P72 + n] = __float2bfloat16_rn(d);
                s.dZ2T[n * P72 + m] = __float2bfloat16_rn(d);
            }
        }
        // dW3 += dY^T A2 (16 x 64 -> rows o < nc), tiles (0, n0) for n0 = warp*16, +8
#pragma unroll
        for (int q = 0; q < 2; ++q) warp_tile(gW3[q], s.dYT, P72, 0, s.A2T, P72, warp * 16 + q * 8, TS);
        __syncthreads();
        // dZ1 = (dZ2 W2) * gelu'(Z1), kept transposed only
        for (int q = 0; q < 8; ++q) {
            const int tl = warp * 8 + q, m0 = (tl >> 3) * 16, n0 = (tl & 7) * 8;
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            warp_tile(acc, s.dZ2, P72, m0, s.W2T, P72, n0, H);
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int m = m0 + g + (r >> 1) * 8, n = n0 + 2 * t + (r & 1);
                s.dZ1T[n * P72 + m] = __float2bfloat16_rn(acc[r] * s.D1[m * H + n]);
            }
        }
        // dW2 += dZ2^T A1 (64 x 64)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int tl = warp * 8 + q, m0 = (tl >> 3) * 16, n0 = (tl & 7) * 8;
            warp_tile(gW2[q], s.dZ2T, P72, m0, s.A1T, P72, n0, TS);
        }
        __syncthreads();
        // dW1 += dZ1^T X (64 x 16): tiles m0 = warp*16, n0 = 0, 8
#pragma unroll
        for (int q = 0; q < 2; ++q) warp_tile(gW1[q], s.dZ1T, P72, warp * 16, s.XT, P72, q * 8, TS);
        // bias gradients: column sums (FP32 from the bf16 tiles' sources)
        for (int h = threadIdx.x; h < 2 * H + nc; h += blockDim.x) {
            float acc = 0.f;
            if (h < H) { for (int m = 0; m < TS; ++m) acc += __bfloat162float(s.dZ1T[h * P72 + m]); }
            else if (h < 2 * H) { for (int m = 0; m < TS; ++m) acc += __bfloat162float(s.dZ2T[(h - H) * P72 + m]); }
            else { for (int m = 0; m < TS; ++m) acc += __bfloat162float(s.dYT[(h - 2 * H) * P72 + m]); }
            s.db[h] += acc;
        }
        __syncthreads();
    }
    // write this block's partial gradient in the layout W1 b1 W2 b2 W3 b3
    float* out = part + (int64_t)blockIdx.x * (n_params + 1);
    const int oW1 = 0, ob1 = H * nc, oW2 = ob1 + H, ob2 = oW2 + H * H, oW3 = ob2 + H, ob3 = oW3 + nc * H;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int tl = warp * 8 + q, m0 = (tl >> 3) * 16, n0 = (tl & 7) * 8;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int m = m0 + g + (r >> 1) * 8, n = n0 + 2 * t + (r & 1);
            out[oW2 + m * H + n] = gW2[q][r];
        }
    }
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int o = g + (r >> 1) * 8, h = warp * 16 + q * 8 + 2 * t + (r & 1);
            if (o < nc) out[oW3 + o * H + h] = gW3[q][r];
            const int hh = warp * 16 + g + (r >> 1) * 8, k = q * 8 + 2 * t + (r & 1);
            if (k < nc) out[oW1 + hh * nc + k] = gW1[q][r];
        }
    for (int h = threadIdx.x; h < 2 * H + nc; h += blockDim.x) {
        if (h < H) out[ob1 + h] = s.db[h];
        else if (h < 2 * H) out[ob2 + h - H] = s.db[h];
        else out[ob3 + h - 2 * H] = s.db[h];
    }
    s.loss[threadIdx.x] = lsum;
    __syncthreads();
    if (threadIdx.x == 0) {
        float l = 0.f;
        for (int i = 0; i < (int)blockDim.x; ++i) l += s.loss[i];
        out[n_params] = l;
    }
}

// Sum block partials in index order; optionally take an Adam step and
// refresh the BF16 operand copies.
__global__ void mlp_update_kernel(MlpDev w, int nc, float* master, float* m1, float* m2, const float* part,
                                  int nblocks, int n_params, float* grad_out, float lr, float b1c, float b2c,
                                  int do_step) {
    const int oW1 = 0, ob1 = H * nc, oW2 = ob1 + H, ob2 = oW2 + H * H, oW3 = ob2 + H, ob3 = oW3 + nc * H;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= n_params; p += gridDim.x * blockDim.x) {
        float gsum = 0.f;
        for (int b = 0; b < nblocks; ++b) gsum += part[(int64_t)b * (n_params + 1) + p];
        if (grad_out) grad_out[p] = gsum;
        if (p == n_params || !do_step) continue;
        const float beta1 = 0.9f, beta2 = 0.999f, eps = 1e-8f;
        const float mm = beta1 * m1[p] + (1.f - beta1) * gsum;
        const float vv = beta2 * m2[p] + (1.f - beta2) * gsum * gsum;
        m1[p] = mm; m2[p] = vv;
        const float upd = lr * (mm / b1c) / (sqrtf(vv / b2c) + eps);
        const float val = master[p] - upd;
        master[p] = val;
        const __nv_bfloat16 bv = __float2bfloat16_rn(val);
        if (p < ob1) { const int h = p / nc, k = p - h * nc; w.W1[h * P24 + k] = bv; }
        else if (p < oW2) w.b[p - ob1] = val;
        else if (p < ob2) { const int o = (p - oW2) / H, i = (p - oW2) - o * H; w.W2[o * P72 + i] = bv; w.W2T[i * P72 + o] = bv; }
        else if (p < oW3) w.b[H + p - ob2] = val;
        else if (p < ob3) { const int o = (p - oW3) / H, h = (p - oW3) - o * H; w.W3[o * P72 + h] = bv; w.W3T[h * P24 + o] = bv; }
        else w.b[2 * H + p - ob3] = val;
    }
}

// Prediction of x0 = log10 T + v for a batch, FP64 in and out.  mode 0:
// inputs are totals (T, FP64) and outputs logfree; mode 1: raw standardised
// FP32 network inputs/outputs (for tests).
__global__ void __launch_bounds__(MLP_THREADS) mlp_predict_kernel(MlpDev w, int nc, const double* totals,
                                                                  double* logfree, const float* xin, float* yout,
                                                                  int64_t n) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmemFwd& s = *reinterpret_cast<MlpSmemFwd*>(smem_raw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    load_weights(s, w, nc);
    __shared__ float nrm[4 * CL_MAX_COMP];
    for (int i = threadIdx.x; i < 4 * nc; i += blockDim.x) nrm[i] = w.norm[i];
    for (int i = threadIdx.x; i < TS * P24; i += blockDim.x) s.X[i] = __float2bfloat16_rn(0.f);
    __syncthreads();
    const int64_t ntiles = (n + TS - 1) / TS;
    for (int64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t s0 = tile * TS;
        const int valid = (int)min((int64_t)TS, n - s0);
        for (int i = threadIdx.x; i < TS * nc; i += blockDim.x) {
            const int m = i / nc, k = i - m * nc;
            float v = 0.f;
            if (m < valid) {
                if (totals) v = (float)((log10(fmax(totals[(s0 + m) * nc + k], 1e-30)) - nrm[k]) / nrm[nc + k]);
                else v = xin[(s0 + m) * nc + k];
            }
            s.X[m * P24 + k] = __float2bfloat16_rn(v);
        }
        __syncthreads();
        float yf[1][4];
        mlp_forward_tile<false>(s, nc, yf);
        const int m0 = warp * 16;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const int m = m0 + g + (r >> 1) * 8, k = 2 * t + (r & 1);
            if (k >= nc || m >= valid) continue;
            if (totals) {
                const double u = log10(fmax(totals[(s0 + m) * nc + k], 1e-30));
                const double v = (double)yf[0][r] * nrm[3 * nc + k] + nrm[2 * nc + k];
                logfree[(s0 + m) * nc + k] = fmin(fmax(u + v, -30.0), 1.0);
            } else {
                yout[(s0 + m) * nc + k] = yf[0][r];
            }
        }
        __syncthreads();
    }
}

// The same inference on the fifth-generation tensor core: 128 samples per
// tile (one per thread, M = 128), the three layers as tcgen05.mma chains on
// shared-memory operands (layer 1 K = 16, layers 2 and 3 K = 64 in four
// MMAs; N = 64, 64, 16) accumulating in 64 TMEM columns, each layer's GELU
// epilogue reading its row from TMEM and writing the next layer's BF16
// operand.  Operands, activations and accumulation are those of
// mlp_predict_kernel (BF16 in, FP32 accumulate, BF16 activations); only the
// order of the FP32 sums differs.  One thread issues the MMAs; completion is
// an mbarrier phase per layer, each wait bounded (on a timeout the kernel
// sets *err and stops after freeing its TMEM).
constexpr int TC_TS = 128, TC_THREADS = 128, TC_COLS = 64;

struct MlpSmemTc {
    alignas(128) unsigned char X[TC_TS * KP * 2];    // [128][16] K-major core matrices
    alignas(128) unsigned char A[TC_TS * H * 2];     // [128][64]
    alignas(128) unsigned char W1[H * KP * 2];       // [64][16]
    alignas(128) unsigned char W2[H * H * 2];        // [64][64]
    alignas(128) unsigned char W3[16 * H * 2];       // [16][64], rows >= nc zero
    float b[2 * H + 16];
    float nrm[4 * CL_MAX_COMP];
    alignas(8) unsigned long long bar;
    uint32_t tmem;
};

__device__ __forceinline__ void tc_put_bf16(unsigned char* tile, int row, int k, int kch, float v) {
    *reinterpret_cast<__nv_bfloat16*>(tile + umma_off(row, k, kch)) = __float2bfloat16_rn(v);
}

// GELU of 16 columns of this thread's row plus bias, into the next operand
__device__ __forceinline__ void tc_gelu16(unsigned char* A, int row, int n0, const float* acc, const float* bias) {
    uint32_t w[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) w[j] = pack_bf16(gelu(acc[2 * j] + bias[n0 + 2 * j]), gelu(acc[2 * j + 1] + bias[n0 + 2 * j + 1]));
    *reinterpret_cast<uint4*>(A + umma_off(row, n0, H / 8)) = make_uint4(w[0], w[1], w[2], w[3]);
    *reinterpret_cast<uint4*>(A + umma_off(row, n0 + 8, H / 8)) = make_uint4(w[4], w[5], w[6], w[7]);
}

__global__ void __launch_bounds__(TC_THREADS) mlp_predict_tc_kernel(MlpDev w, int nc, const double* totals,
                                                                   double* logfree, const float* xin, float* yout,
                                                                   int64_t n, unsigned int* err) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    MlpSmemTc& s = *reinterpret_cast<MlpSmemTc*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    // weights into the K-major core-matrix layout, biases, normalisation
    for (int i = tid; i < H * KP; i += TC_THREADS) {
        const int r = i / KP, k = i - r * KP;
        *reinterpret_cast<__nv_bfloat16*>(s.W1 + umma_off(r, k, KP / 8)) = w.W1[r * P24 + k];
    }
    for (int i = tid; i < H * H; i += TC_THREADS) {
        const int r = i / H, k = i - r * H;
        *reinterpret_cast<__nv_bfloat16*>(s.W2 + umma_off(r, k, H / 8)) = w.W2[r * P72 + k];
    }
    for (int i = tid; i < 16 * H; i += TC_THREADS) {
        const int r = i / H, k = i - r * H;
        *reinterpret_cast<__nv_bfloat16*>(s.W3 + umma_off(r, k, H / 8)) =
            r < nc && r < 8 ? w.W3[r * P72 + k] : __float2bfloat16_rn(0.f);
    }
    for (int i = tid; i < 2 * H + 16; i += TC_THREADS) s.b[i] = i < 2 * H + nc ? w.b[i] : 0.f;
    for (int i = tid; i < 4 * nc; i += TC_THREADS) s.nrm[i] = w.norm[i];
    const uint32_t bar = smem_u32(&s.bar);
    if (tid == 0) mbar_init(bar, 1);
    if (warp == 0) tmem_alloc(smem_u32(&s.tmem), TC_COLS);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t aX = smem_u32(s.X), aA = smem_u32(s.A), aW1 = smem_u32(s.W1), aW2 = smem_u32(s.W2),
                   aW3 = smem_u32(s.W3);
    constexpr int kLimit = 1 << 20;
    uint32_t phase = 0;
    bool ok = true;
    const int64_t ntiles = (n + TC_TS - 1) / TC_TS;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int64_t s0 = tile * TC_TS;
        const int m = tid;                       // this thread's sample and TMEM lane
        const bool valid = s0 + m < n;
        // layer-1 operand: the standardised inputs, zero beyond nc and n
        {
            uint32_t wv[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                float v2[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = 2 * j + h;
                    float v = 0.f;
                    if (valid && k < nc) {
                        if (totals) v = (float)((log10(fmax(totals[(s0 + m) * nc + k], 1e-30)) - s.nrm[k]) / s.nrm[nc + k]);
                        else v = xin[(s0 + m) * nc + k];
                    }
                    v2[h] = v;
                }
                wv[j] = pack_bf16(v2[0], v2[1]);
            }
            *reinterpret_cast<uint4*>(s.X + umma_off(m, 0, KP / 8)) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
            *reinterpret_cast<uint4*>(s.X + umma_off(m, 8, KP / 8)) = make_uint4(wv[4], wv[5], wv[6], wv[7]);
        }
        // three layers: operand ready -> one thread issues -> commit -> all wait -> epilogue
#pragma unroll 1
        for (int layer = 0; layer < 3; ++layer) {
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                if (layer == 0) {
                    umma_bf16(tmem, umma_desc(aX, 0, KP / 8), umma_desc(aW1, 0, KP / 8), umma_idesc_bf16(H), 0);
                } else {
                    const uint32_t wB = layer == 1 ? aW2 : aW3;
                    const uint32_t id = umma_idesc_bf16(layer == 1 ? H : 16);
#pragma unroll
                    for (int kb = 0; kb < H / 16; ++kb)
                        umma_bf16(tmem, umma_desc(aA, kb, H / 8), umma_desc(wB, kb, H / 8), id, kb > 0);
                }
                umma_commit(bar);
            }
            // every thread leaves together if any wait timed out
            if (!__syncthreads_and(mbar_wait(bar, phase & 1u, kLimit))) { ok = false; break; }
            ++phase;
            tc_fence_after();
            if (layer < 2) {
                const float* bias = s.b + layer * H;
#pragma unroll
                for (int c = 0; c < H / 16; ++c) {
                    float acc[16];
                    tmem_ld16(lane_addr + (uint32_t)(16 * c), acc);
                    tc_gelu16(s.A, m, 16 * c, acc, bias);
                }
            } else {
                float acc[16];
                tmem_ld16(lane_addr, acc);
                if (valid) {
                    for (int k = 0; k < nc; ++k) {
                        const float y = acc[k] + s.b[2 * H + k];
                        if (totals) {
                            const double u = log10(fmax(totals[(s0 + m) * nc + k], 1e-30));
                            const double v = (double)y * s.nrm[3 * nc + k] + s.nrm[2 * nc + k];
                            logfree[(s0 + m) * nc + k] = fmin(fmax(u + v, -30.0), 1.0);
                        } else {
                            yout[(s0 + m) * nc + k] = y;
                        }
                    }
                }
            }
        }
    }
    if (!ok) {
        // one more bounded wait for MMAs still in flight before the TMEM goes
        mbar_wait(bar, phase & 1u, kLimit);
        if (tid == 0) atomicOr(err, 1u);
    }
    // every thread's TMEM reads are done before the allocating warp frees it
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, TC_COLS);
}

// ---------------------------------------------------------------- Newton batch
template <int NC>
__global__ void newton_first_kernel(EqDev e, const double* totals, const double* cold_species, double* logfree,
                                     int32_t* iters, uint8_t* status, int64_t n, int start, int limit,
                                     double tol, int64_t* fail_list, unsigned long long* fail_count) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
        double T[NC], x[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = totals[k * NC + j];
        if (start == CL_EQ_START_COLD) eq_cold_start<NC>(e, cold_species + k * e.ns, x);
        else {
#pragma unroll
            for (int j = 0; j < NC; ++j) x[j] = logfree[k * NC + j];
        }
        int conv = 0;
        const int it = eq_newton<NC>(e, T, x, limit, tol, &conv);
#pragma unroll
        for (int j = 0; j < NC; ++j) logfree[k * NC + j] = x[j];
        if (iters) iters[k] = it;
        if (conv) { if (status) status[k] = 0; }
        else if (start == CL_EQ_START_COLD || !fail_list) { if (status) status[k] = 2; }
        else {
            const unsigned long long slot = atomicAdd(fail_count, 1ull);
            fail_list[slot] = k;
        }
    }
}

template <int NC>
__global__ void newton_fallback_kernel(EqDev e, const double* totals, const double* cold_species, double* logfree,
                                        int32_t* iters, uint8_t* status, const int64_t* fail_list,
                                        const unsigned long long* fail_count, int limit, double tol) {
    const int64_t cnt = (int64_t)*fail_count;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += stride) {
        const int64_t k = fail_list[q];
        double T[NC], x[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = totals[k * NC + j];
        eq_cold_start<NC>(e, cold_species + k * e.ns, x);
        int conv = 0;
        const int it = eq_newton<NC>(e, T, x, limit, tol, &conv);
#pragma unroll
        for (int j = 0; j < NC; ++j) logfree[k * NC + j] = x[j];
        if (iters) iters[k] += it;
        if (status) status[k] = conv ? 1 : 2;
    }
}

// One pass of the bucketed solve: every listed voxel (all n when `in_list` is
// null) runs at most `budget` Newton iterations from its stored x (mode 0), the
// reference's cold start (mode 1) or the given start (mode 2); converged voxels
// get status `ok_status`, the others are appended to `out_list` for the next
// pass, or get status 2 when this is the last pass.  Newton keeps no state
// besides x, so a solve split over passes is the same solve; a solve that
// stopped early (stop_mark) is carried through the remaining passes of its
// phase without running, as the unsplit solve would have ended there.
// lists at most this long are solved one warp per system (newton_pass_warp_kernel)
constexpr int64_t kWarpPassMax = 4096;

template <int NC>
__global__ void __launch_bounds__(128, 4) newton_pass_kernel(EqDev e, const double* totals, const double* cold_species, double* logfree,
                                   int32_t* iters, uint8_t* status, const int64_t* in_list,
                                   const unsigned long long* in_count, int64_t n, int mode, int budget, double tol,
                                   int ok_status, int last, int64_t* out_list, unsigned long long* out_count,
                                   uint8_t* stop_mark) {
    const int64_t cnt = in_list ? (int64_t)*in_count : n;
    if (cnt <= kWarpPassMax) return;           // the warp-per-solve pass takes short lists
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < cnt; q += stride) {
        const int64_t k = in_list ? in_list[q] : q;
        if (mode == 0 && stop_mark[k]) {
            if (last) { if (status) status[k] = 2; }
            else out_list[atomicAdd(out_count, 1ull)] = k;
            continue;
        }
        double T[NC], x[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = totals[k * NC + j];
        if (mode == 1) eq_cold_start<NC>(e, cold_species + k * e.ns, x);
        else {
#pragma unroll
            for (int j = 0; j < NC; ++j) x[j] = logfree[k * NC + j];
        }
        int conv = 0, stopped = 0;
        const int it = eq_newton<NC>(e, T, x, budget, tol, &conv, &stopped);
#pragma unroll
        for (int j = 0; j < NC; ++j) logfree[k * NC + j] = x[j];
        stop_mark[k] = (uint8_t)(stopped && !conv);
        if (iters) iters[k] = (mode == 0 ? iters[k] : (mode == 1 && in_list ? iters[k] : 0)) + it;
        if (conv) { if (status) status[k] = (uint8_t)ok_status; }
        else if (last) { if (status) status[k] = 2; }
        else out_list[atomicAdd(out_count, 1ull)] = k;
    }
}

template <int NC>
__global__ void newton_pass_warp_kernel(EqDev e, const double* totals, const double* cold_species, double* logfree,
                                   int32_t* iters, uint8_t* status, const int64_t* in_list,
                                   const unsigned long long* in_count, int64_t n, int mode, int budget, double tol,
                                   int ok_status, int last, int64_t* out_list, unsigned long long* out_count,
                                   uint8_t* stop_mark) {
    const int64_t cnt = in_list ? (int64_t)*in_count : n;
    if (cnt > kWarpPassMax) return;            // long lists: newton_pass_kernel
    const bool lead = (threadIdx.x & 31) == 0;
    const int64_t stride = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t q = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < cnt; q += stride) {
        const int64_t k = in_list ? in_list[q] : q;
        if (mode == 0 && stop_mark[k]) {
            if (lead) {
                if (last) { if (status) status[k] = 2; }
                else out_list[atomicAdd(out_count, 1ull)] = k;
            }
            continue;
        }
        double T[NC], x[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = totals[k * NC + j];
        if (mode == 1) eq_cold_start<NC>(e, cold_species + k * e.ns, x);
        else {
#pragma unroll
            for (int j = 0; j < NC; ++j) x[j] = logfree[k * NC + j];
        }
        int conv = 0, stopped = 0;
        const int it = eq_newton_warp<NC>(e, T, x, budget, tol, &conv, &stopped);
        __syncwarp();                          // every lane has read iters[k] / stop_mark[k]
        if (!lead) continue;
#pragma unroll
        for (int j = 0; j < NC; ++j) logfree[k * NC + j] = x[j];
        stop_mark[k] = (uint8_t)(stopped && !conv);
        if (iters) iters[k] = (mode == 0 ? iters[k] : (mode == 1 && in_list ? iters[k] : 0)) + it;
        if (conv) { if (status) status[k] = (uint8_t)ok_status; }
        else if (last) { if (status) status[k] = 2; }
        else out_list[atomicAdd(out_count, 1ull)] = k;
    }
}

}  // namespace cl

using namespace cl;

// calculate_species_concentrations (part4_eqsolver.hh:1187-1214) per entry:
// one PCF + Anderson solve per thread from the entry's species row.
template <int NC>
__global__ void __launch_bounds__(128) pcf_batch_kernel(const __grid_constant__ EqDev e, const double* in,
                                                        double* out, int32_t* iters, uint8_t* conv, int64_t n,
                                                        int max_iter, double tol, unsigned long long* nonconv) {
    unsigned long long miss = 0;
    const int ns = e.ns;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        const double* c = in + k * ns;
        double T[NC], x[NC];
        pcf_totals_and_start<NC>(e, c, 1, T, x);
        int cv = 0;
        const int it = eq_pcf<NC>(e, T, c, 1, x, max_iter, tol, e.depth, &cv);
        for (int i = 0; i < ns; ++i) {
            double v = e.active[i] ? pcf_species<NC>(e, i, x, c[i]) : pcf_passive(c[i]);
            if (isnan(v) || isinf(v)) v = pcf_passive(c[i]);
            out[k * ns + i] = pcf_max(pcf_min(v, 10.0), 1e-30);
        }
        if (iters) iters[k] = it;
        if (conv) conv[k] = (uint8_t)cv;
        miss += cv ? 0 : 1;
    }
    for (int o = 16; o > 0; o >>= 1) miss += __shfl_down_sync(0xffffffffu, miss, o);
    if ((threadIdx.x & 31) == 0 && miss) atomicAdd(nonconv, miss);
}

struct cl_eq_solver {
    cl_eq_system sys;
    EqDev e;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int nc = 0, n_params = 0;
    MlpDev w{};
    float* master = nullptr;   // FP32 parameters (oracle layout)
    float* m1 = nullptr;
    float* m2 = nullptr;
    float* part = nullptr;     // per-block partial gradients
    int part_blocks = 0;
    float* grad = nullptr;     // n_params + 1 (loss)
    bool trained = false;
    int64_t* fail_list = nullptr;     // ping-pong lists of the bucketed solve
    int64_t* fail_list2 = nullptr;
    uint8_t* stop_mark = nullptr;     // solves that stopped early in the current phase
    int64_t fail_cap = 0;
    unsigned long long* fail_count = nullptr;   // two counters
    int net_path = CL_EQ_NET_TCGEN05;           // the network's inference kernel
    unsigned int* tc_err = nullptr;             // set by the tcgen05 kernel on a wait timeout
    unsigned long long* pcf_count = nullptr;    // PCF solves that did not converge
    uint64_t adam_t = 0;
    // tableaux beyond the one-thread solver (more than 5 components or more
    // species than kEqDevSpecies): the warp solver of speciation_large.cu on a
    // device copy of the tableau; no network, no PCF
    bool large = false;
    LgTableau lg{};
    double* lg_stoich = nullptr;
    double* lg_logk = nullptr;
    uint8_t* lg_active = nullptr;
};

// entry points that need the network or the one-thread solvers refuse a large tableau
static bool refuse_large(const cl_eq_solver* s, const char* what) {
    if (!s->large) return false;
    set_error(std::string(what) + ": not available for tableaux above 5 components or " +
              std::to_string(kEqDevSpecies) + " species (the batch Newton solve is)");
    return true;
}

int cl::eq_solver_network(cl_eq_solver* s, const float** master, const float** norm, int* trained) {
    if (!s || s->large) return CL_ERR_ARG;
    *master = s->master;
    *norm = s->w.norm;
    *trained = s->trained ? 1 : 0;
    return CL_OK;
}

static cl_eq_solver* create_large(const cl_eq_system* sys, void* stream, int* status) {
    const int nc = sys->n_comp, ns = sys->n_species;
    cl_eq_solver* s = new cl_eq_solver();
    auto fail = [&](int st) { if (status) *status = st; cl_eq_destroy(s); return (cl_eq_solver*)nullptr; };
    s->sys = *sys;
    s->nc = nc;
    s->large = true;
    if (stream) s->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(CL_ERR_CUDA);
        s->own_stream = true;
    }
    std::vector<double> St((size_t)ns * nc), lk(ns);
    std::vector<uint8_t> act(ns, 0);
    for (int i = 0; i < ns; ++i) {
        lk[i] = sys->logk[i];
        for (int j = 0; j < nc; ++j) {
            const double v = sys->stoich[i][j];
            St[(size_t)i * nc + j] = v;
            if (v > 1e-10 || v < -1e-10) act[i] = 1;
        }
    }
    cudaError_t e = cudaMalloc(&s->lg_stoich, sizeof(double) * St.size());
    if (e == cudaSuccess) e = cudaMalloc(&s->lg_logk, sizeof(double) * ns);
    if (e == cudaSuccess) e = cudaMalloc(&s->lg_active, ns);
    if (e == cudaSuccess) e = cudaMalloc(&s->fail_count, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->lg_stoich, St.data(), sizeof(double) * St.size(), cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->lg_logk, lk.data(), sizeof(double) * ns, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->lg_active, act.data(), ns, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cl_eq_create"));
    s->lg.nc = nc;
    s->lg.ns = ns;
    s->lg.stoich = s->lg_stoich;
    s->lg.logk = s->lg_logk;
    s->lg.active = s->lg_active;
    for (int j = 0; j < CL_MAX_COMP; ++j) s->lg.comp_species[j] = j < nc ? sys->comp_species[j] : -1;
    if (status) *status = CL_OK;
    return s;
}

static size_t mlp_smem_bytes() { return sizeof(MlpSmem); }
static size_t mlp_fwd_smem_bytes() { return sizeof(MlpSmemFwd); }

// the network's inference on the selected tensor-core path (mode as
// mlp_predict_kernel: totals -> logfree, or raw xin -> yout)
static int predict_launch(cl_eq_solver* s, const double* totals, double* logfree, const float* xin, float* yout,
                          int64_t n) {
    if (s->net_path == CL_EQ_NET_TCGEN05) {
        mlp_predict_tc_kernel<<<grid_for((n + TC_TS - 1) / TC_TS, 1, 148 * 4), TC_THREADS, sizeof(MlpSmemTc),
                                s->stream>>>(s->w, s->nc, totals, logfree, xin, yout, n, s->tc_err);
        CL_LAUNCH_CHECK("mlp_predict_tc_kernel");
    } else {
        mlp_predict_kernel<<<grid_for((n + TS - 1) / TS, 1, 148 * 6), MLP_THREADS, mlp_fwd_smem_bytes(), s->stream>>>(
            s->w, s->nc, totals, logfree, xin, yout, n);
        CL_LAUNCH_CHECK("mlp_predict_kernel");
    }
    return CL_OK;
}

// a tcgen05 inference that timed out waiting for its MMAs (read after a
// synchronisation of the solver's stream); clears the flag
static int tc_error(cl_eq_solver* s, const char* where) {
    unsigned int v = 0;
    CL_CUDA(cudaMemcpy(&v, s->tc_err, sizeof(v), cudaMemcpyDeviceToHost));
    if (!v) return CL_OK;
    CL_CUDA(cudaMemset(s->tc_err, 0, sizeof(v)));
    set_error(std::string(where) + ": the tensor-core inference timed out waiting for its MMAs");
    return CL_ERR_CUDA;
}

static int eq_ensure_fail(cl_eq_solver* s, int64_t n) {
    if (s->fail_cap >= n) return CL_OK;
    if (s->fail_list) cudaFree(s->fail_list);
    if (s->fail_list2) cudaFree(s->fail_list2);
    if (s->stop_mark) cudaFree(s->stop_mark);
    s->fail_list = s->fail_list2 = nullptr;
    s->stop_mark = nullptr;
    CL_CUDA(cudaMalloc(&s->fail_list, sizeof(int64_t) * (size_t)std::max<int64_t>(n, 1)));
    CL_CUDA(cudaMalloc(&s->fail_list2, sizeof(int64_t) * (size_t)std::max<int64_t>(n, 1)));
    CL_CUDA(cudaMalloc(&s->stop_mark, (size_t)std::max<int64_t>(n, 1)));
    s->fail_cap = n;
    return CL_OK;
}

// Iteration budgets of the bucketed passes: short passes first (most solves
// finish there), then doubling, summing to `total`.
static std::vector<int> bucket_budgets(int total, int first) {
    std::vector<int> b;
    int used = 0, next = std::max(1, first);
    while (used < total) {
        const int take = std::min(next, total - used);
        b.push_back(take);
        used += take;
        if (b.size() >= 2) next *= 2;
    }
    return b;
}

template <int NC>
static int bucketed_solve(cl_eq_solver* s, const double* T, const double* cold, double* x, int32_t* it,
                          uint8_t* st, int64_t n, int start) {
    const int blocks = grid_for(n, 128, 148 * 16);
    unsigned long long* cnt[2] = {s->fail_count, s->fail_count + 1};
    int64_t* lists[2] = {s->fail_list, s->fail_list2};
    int cur = -1;   // list holding the voxels still to solve (-1: all n)
    auto pass = [&](int mode, int budget, int ok_status, bool last) -> int {
        const int out = (cur == 0) ? 1 : 0;
        CL_CUDA(cudaMemsetAsync(cnt[out], 0, sizeof(unsigned long long), s->stream));
        // both kernels read the list length on the device and only one works
        if (cur >= 0 || n > kWarpPassMax) {
            newton_pass_kernel<NC><<<blocks, 128, 0, s->stream>>>(
                s->e, T, cold, x, it, st, cur < 0 ? nullptr : lists[cur], cur < 0 ? nullptr : cnt[cur], n, mode,
                budget, s->sys.tol, ok_status, last ? 1 : 0, lists[out], cnt[out], s->stop_mark);
            CL_LAUNCH_CHECK("newton_pass_kernel");
        }
        if (cur >= 0 || n <= kWarpPassMax) {
            newton_pass_warp_kernel<NC><<<(int)(kWarpPassMax * 32 / 128), 128, 0, s->stream>>>(
                s->e, T, cold, x, it, st, cur < 0 ? nullptr : lists[cur], cur < 0 ? nullptr : cnt[cur], n, mode,
                budget, s->sys.tol, ok_status, last ? 1 : 0, lists[out], cnt[out], s->stop_mark);
            CL_LAUNCH_CHECK("newton_pass_warp_kernel");
        }
        cur = out;
        return CL_OK;
    };
    int r = CL_OK;
    std::vector<int> cold_b = bucket_budgets(s->sys.max_iter, 3);
    if (start == CL_EQ_START_COLD) {
        for (size_t i = 0; i < cold_b.size(); ++i)
            if ((r = pass(i == 0 ? 1 : 0, cold_b[i], 0, i + 1 == cold_b.size()))) return r;
        return CL_OK;
    }
    // warm start with warm_iter iterations in short passes, then the cold
    // restart for the misses
    const bool fallback = cold != nullptr;
    std::vector<int> warm_b = bucket_budgets(s->sys.warm_iter, 2);
    for (size_t i = 0; i < warm_b.size(); ++i)
        if ((r = pass(i == 0 ? 2 : 0, warm_b[i], 0, !fallback && i + 1 == warm_b.size()))) return r;
    if (!fallback) return CL_OK;
    for (size_t i = 0; i < cold_b.size(); ++i)
        if ((r = pass(i == 0 ? 1 : 0, cold_b[i], 1, i + 1 == cold_b.size()))) return r;
    return CL_OK;
}

static int upload_params(cl_eq_solver* s, const float* host) {
    // write master, reset Adam, rebuild BF16 copies through the update kernel with lr = 0
    const int np = s->n_params;
    CL_CUDA(cudaMemcpyAsync(s->master, host, sizeof(float) * np, cudaMemcpyHostToDevice, s->stream));
    CL_CUDA(cudaMemsetAsync(s->m1, 0, sizeof(float) * np, s->stream));
    CL_CUDA(cudaMemsetAsync(s->m2, 0, sizeof(float) * np, s->stream));
    CL_CUDA(cudaMemsetAsync(s->part, 0, sizeof(float) * (np + 1), s->stream));
    mlp_update_kernel<<<64, 256, 0, s->stream>>>(s->w, s->nc, s->master, s->m1, s->m2, s->part, 1, np, nullptr,
                                                 0.f, 1.f, 1.f, 1);
    CL_LAUNCH_CHECK("mlp_update_kernel");
    CL_CUDA(cudaMemsetAsync(s->m1, 0, sizeof(float) * np, s->stream));
    CL_CUDA(cudaMemsetAsync(s->m2, 0, sizeof(float) * np, s->stream));
    return CL_OK;
}

extern "C" {

cl_eq_solver* cl_eq_create(const cl_eq_system* sys, void* stream, int* status) {
    auto fail = [&](int st, cl_eq_solver* s) { if (status) *status = st; cl_eq_destroy(s); return (cl_eq_solver*)nullptr; };
    if (!sys || sys->n_comp < 1 || sys->n_comp > CL_MAX_COMP || sys->n_species < sys->n_comp ||
        sys->n_species > CL_MAX_SPECIES) {
        set_error("speciation batch needs 1.." + std::to_string(CL_MAX_COMP) + " components and n_comp <= n_species <= " +
                  std::to_string(CL_MAX_SPECIES));
        if (status) *status = CL_ERR_ARG;
        return nullptr;
    }
    for (int j = 0; j < sys->n_comp; ++j)
        if (sys->comp_species[j] < -1 || sys->comp_species[j] >= sys->n_species) {
            set_error("comp_species out of range");
            if (status) *status = CL_ERR_ARG;
            return nullptr;
        }
    if (sys->max_iter < 0 || sys->warm_iter < 0) {
        set_error("max_iter and warm_iter must be >= 0");
        if (status) *status = CL_ERR_ARG;
        return nullptr;
    }
    if (sys->n_comp > 5 || sys->n_species > kEqDevSpecies) return create_large(sys, stream, status);
    if ((sys->solver != CL_EQ_SOLVER_NEWTON && sys->solver != CL_EQ_SOLVER_PCF) || sys->anderson_depth < 0 ||
        sys->anderson_depth > kPcfMaxDepth) {
        set_error("unknown equilibrium solver, or anderson_depth outside 0..8");
        if (status) *status = CL_ERR_ARG;
        return nullptr;
    }
    cl_eq_solver* s = new cl_eq_solver();
    s->sys = *sys;
    eqdev_from_system(*sys, s->e);
    s->nc = sys->n_comp;
    s->n_params = H * s->nc + H + H * H + H + s->nc * H + s->nc;
    if (stream) s->stream = (cudaStream_t)stream;
    else {
        if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess) return fail(CL_ERR_CUDA, s);
        s->own_stream = true;
    }
    const int np = s->n_params;
    s->part_blocks = 148;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) { if (e == cudaSuccess) e = cudaMalloc(p, bytes); if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s->stream); };
    A((void**)&s->w.W1, sizeof(__nv_bfloat16) * H * P24);
    A((void**)&s->w.W2, sizeof(__nv_bfloat16) * H * P72);
    A((void**)&s->w.W2T, sizeof(__nv_bfloat16) * H * P72);
    A((void**)&s->w.W3, sizeof(__nv_bfloat16) * 8 * P72);
    A((void**)&s->w.W3T, sizeof(__nv_bfloat16) * H * P24);
    A((void**)&s->w.b, sizeof(float) * (2 * H + 8));
    A((void**)&s->w.norm, sizeof(float) * 4 * CL_MAX_COMP);
    A((void**)&s->master, sizeof(float) * np);
    A((void**)&s->m1, sizeof(float) * np);
    A((void**)&s->m2, sizeof(float) * np);
    A((void**)&s->part, sizeof(float) * (size_t)s->part_blocks * (np + 1));
    A((void**)&s->grad, sizeof(float) * (np + 1));
    A((void**)&s->fail_count, 2 * sizeof(unsigned long long));
    A((void**)&s->tc_err, sizeof(unsigned int));
    A((void**)&s->pcf_count, sizeof(unsigned long long));
    if (e != cudaSuccess) return fail(cuda_fail(e, "cl_eq_create"), s);
    if (cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_smem_bytes()) != cudaSuccess ||
        cudaFuncSetAttribute(mlp_predict_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mlp_fwd_smem_bytes()) != cudaSuccess ||
        cudaFuncSetAttribute(mlp_predict_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(MlpSmemTc)) != cudaSuccess)
        return fail(cuda_fail(cudaGetLastError(), "cudaFuncSetAttribute(mlp)"), s);
    // default initialisation: Glorot-uniform weights, zero biases, identity normalisation
    std::vector<float> p(np, 0.f);
    std::mt19937_64 rng(12345);
    auto glorot = [&](int off, int fan_out, int fan_in) {
        const float a = std::sqrt(6.f / (fan_in + fan_out));
        std::uniform_real_distribution<float> U(-a, a);
        for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = U(rng);
    };
    glorot(0, H, s->nc);
    glorot(H * s->nc + H, H, H);
    glorot(H * s->nc + H + H * H + H, s->nc, H);
    std::vector<float> norm(4 * CL_MAX_COMP, 0.f);
    for (int j = 0; j < s->nc; ++j) { norm[s->nc + j] = 1.f; norm[3 * s->nc + j] = 1.f; }
    if (cudaMemcpyAsync(s->w.norm, norm.data(), sizeof(float) * norm.size(), cudaMemcpyHostToDevice, s->stream) != cudaSuccess)
        return fail(CL_ERR_CUDA, s);
    int r = upload_params(s, p.data());
    if (r) return fail(r, s);
    if (cudaStreamSynchronize(s->stream) != cudaSuccess) return fail(cuda_fail(cudaGetLastError(), "cl_eq_create"), s);
    if (status) *status = CL_OK;
    return s;
}

int cl_eq_destroy(cl_eq_solver* s) {
    if (!s) return CL_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    void* ptrs[] = {s->w.W1, s->w.W2, s->w.W2T, s->w.W3, s->w.W3T, s->w.b, s->w.norm, s->master, s->m1, s->m2,
                    s->part, s->grad, s->fail_list, s->fail_list2, s->stop_mark, s->fail_count, s->pcf_count,
                    s->lg_stoich, s->lg_logk, s->lg_active, s->tc_err};
    for (void* p : ptrs) if (p) cudaFree(p);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return CL_OK;
}

int cl_eq_param_count(const cl_eq_solver* s, int32_t* count) {
    if (!s || !count) return CL_ERR_ARG;
    *count = s->n_params;
    return CL_OK;
}

int cl_eq_get_params(cl_eq_solver* s, float* host) {
    if (!s || !host) return CL_ERR_ARG;
    if (refuse_large(s, "cl_eq_get_params")) return CL_ERR_ARG;
    CL_CUDA(cudaMemcpyAsync(host, s->master, sizeof(float) * s->n_params, cudaMemcpyDeviceToHost, s->stream));
    CL_CUDA(cudaStreamSynchronize(s->stream));
    return CL_OK;
}

int cl_eq_set_params(cl_eq_solver* s, const float* host) {
    if (!s || !host) return CL_ERR_ARG;
    if (refuse_large(s, "cl_eq_set_params")) return CL_ERR_ARG;
    int r = upload_params(s, host);
    if (r) return r;
    CL_CUDA(cudaStreamSynchronize(s->stream));
    return CL_OK;
}

int cl_eq_solve_device(cl_eq_solver* s, const double* d_totals, const double* d_cold_species, double* d_logfree,
                       int32_t* d_iters, uint8_t* d_status, int64_t n, int32_t start) {
    if (!s || !d_totals || !d_logfree || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (n == 0) return CL_OK;
    if (start == CL_EQ_START_COLD && !d_cold_species) { set_error("cold start needs the species vectors"); return CL_ERR_ARG; }
    if (s->large) {
        if (start != CL_EQ_START_GIVEN && start != CL_EQ_START_COLD) {
            set_error("large tableaux start cold or from a given point");
            return CL_ERR_ARG;
        }
        return lg_solve(s->lg, s->stream, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start,
                        s->sys.max_iter, s->sys.warm_iter, s->sys.tol, s->fail_count);
    }
    if (start == CL_EQ_START_LEARNED) {
        const int rp = predict_launch(s, d_totals, d_logfree, nullptr, nullptr, n);
        if (rp) return rp;
    } else if (start != CL_EQ_START_GIVEN && start != CL_EQ_START_COLD) { set_error("unknown start mode"); return CL_ERR_ARG; }
    int r = eq_ensure_fail(s, n);
    if (r) return r;
    switch (s->nc) {
        case 1: return bucketed_solve<1>(s, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start);
        case 2: return bucketed_solve<2>(s, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start);
        case 3: return bucketed_solve<3>(s, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start);
        case 4: return bucketed_solve<4>(s, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start);
        default: return bucketed_solve<5>(s, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start);
    }
}

int cl_eq_pcf_device(cl_eq_solver* s, const double* d_in, double* d_out, int32_t* d_iters, uint8_t* d_conv,
                     int64_t n) {
    if (!s || !d_in || !d_out || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (refuse_large(s, "cl_eq_pcf_device")) return CL_ERR_ARG;
    if (n == 0) return CL_OK;
    CL_CUDA(cudaMemsetAsync(s->pcf_count, 0, sizeof(unsigned long long), s->stream));
    const int blocks = grid_for(n, 128, 148 * 8);
    const int mi = s->sys.max_iter;
    const double tol = s->sys.tol;
    switch (s->nc) {
        case 1: pcf_batch_kernel<1><<<blocks, 128, 0, s->stream>>>(s->e, d_in, d_out, d_iters, d_conv, n, mi, tol, s->pcf_count); break;
        case 2: pcf_batch_kernel<2><<<blocks, 128, 0, s->stream>>>(s->e, d_in, d_out, d_iters, d_conv, n, mi, tol, s->pcf_count); break;
        case 3: pcf_batch_kernel<3><<<blocks, 128, 0, s->stream>>>(s->e, d_in, d_out, d_iters, d_conv, n, mi, tol, s->pcf_count); break;
        case 4: pcf_batch_kernel<4><<<blocks, 128, 0, s->stream>>>(s->e, d_in, d_out, d_iters, d_conv, n, mi, tol, s->pcf_count); break;
        default: pcf_batch_kernel<5><<<blocks, 128, 0, s->stream>>>(s->e, d_in, d_out, d_iters, d_conv, n, mi, tol, s->pcf_count); break;
    }
    CL_LAUNCH_CHECK("pcf_batch_kernel");
    unsigned long long miss = 0;
    CL_CUDA(cudaMemcpyAsync(&miss, s->pcf_count, sizeof miss, cudaMemcpyDeviceToHost, s->stream));
    CL_CUDA(cudaStreamSynchronize(s->stream));
    return miss ? CL_WARN_NOT_CONVERGED : CL_OK;
}

int cl_eq_pcf_host(cl_eq_solver* s, const double* in, double* out, int32_t* iters, uint8_t* conv, int64_t n) {
    if (!s || !in || !out || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (n == 0) return CL_OK;
    const int ns = s->sys.n_species;
    double *dIn = nullptr, *dOut = nullptr;
    int32_t* dI = nullptr;
    uint8_t* dC = nullptr;
    int r = CL_OK;
    cudaError_t e = cudaMalloc(&dIn, sizeof(double) * n * ns);
    if (e == cudaSuccess) e = cudaMalloc(&dOut, sizeof(double) * n * ns);
    if (e == cudaSuccess) e = cudaMalloc(&dI, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dC, n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dIn, in, sizeof(double) * n * ns, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_pcf_host");
    if (!r) r = cl_eq_pcf_device(s, dIn, dOut, dI, dC, n);
    if (r >= 0) {
        e = cudaMemcpyAsync(out, dOut, sizeof(double) * n * ns, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess && iters) e = cudaMemcpyAsync(iters, dI, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess && conv) e = cudaMemcpyAsync(conv, dC, n, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_pcf_host");
    }
    cudaFree(dIn); cudaFree(dOut); cudaFree(dI); cudaFree(dC);
    return r;
}

int cl_eq_predict_device(cl_eq_solver* s, const double* d_totals, double* d_logfree, int64_t n) {
    if (!s || !d_totals || !d_logfree || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (refuse_large(s, "cl_eq_predict_device")) return CL_ERR_ARG;
    if (n == 0) return CL_OK;
    return predict_launch(s, d_totals, d_logfree, nullptr, nullptr, n);
}

int cl_eq_solve_host(cl_eq_solver* s, const double* totals, const double* cold_species, double* logfree,
                     int32_t* iters, uint8_t* status, int64_t n, int32_t start) {
    if (!s || !totals || !logfree || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (n == 0) return CL_OK;
    const int nc = s->nc, ns = s->sys.n_species;
    double *dT = nullptr, *dC = nullptr, *dX = nullptr;
    int32_t* dI = nullptr;
    uint8_t* dS = nullptr;
    int r = CL_OK;
    cudaError_t e = cudaMalloc(&dT, sizeof(double) * n * nc);
    if (e == cudaSuccess) e = cudaMalloc(&dX, sizeof(double) * n * nc);
    if (e == cudaSuccess && cold_species) e = cudaMalloc(&dC, sizeof(double) * n * ns);
    if (e == cudaSuccess) e = cudaMalloc(&dI, sizeof(int32_t) * n);
    if (e == cudaSuccess) e = cudaMalloc(&dS, n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dT, totals, sizeof(double) * n * nc, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess && cold_species) e = cudaMemcpyAsync(dC, cold_species, sizeof(double) * n * ns, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess && start == CL_EQ_START_GIVEN) e = cudaMemcpyAsync(dX, logfree, sizeof(double) * n * nc, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_solve_host");
    if (!r) r = cl_eq_solve_device(s, dT, dC, dX, dI, dS, n, start);
    // CL_WARN_NOT_CONVERGED still returns every entry's solution and status
    if (r >= 0) {
        e = cudaMemcpyAsync(logfree, dX, sizeof(double) * n * nc, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess && iters) e = cudaMemcpyAsync(iters, dI, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess && status) e = cudaMemcpyAsync(status, dS, n, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_solve_host");
    }
    cudaFree(dT); cudaFree(dC); cudaFree(dX); cudaFree(dI); cudaFree(dS);
    return r;
}

// gradients of one batch (no update), for checks against the FP64 oracle
int cl_eq_grad_host(cl_eq_solver* s, const float* x, const float* y, int32_t n, float* loss, float* grads) {
    if (!s || !x || !y || n <= 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (refuse_large(s, "cl_eq_grad_host")) return CL_ERR_ARG;
    const int nc = s->nc, np = s->n_params;
    float *dx = nullptr, *dy = nullptr;
    CL_CUDA(cudaMalloc(&dx, sizeof(float) * n * nc));
    CL_CUDA(cudaMalloc(&dy, sizeof(float) * n * nc));
    int r = CL_OK;
    cudaError_t e = cudaMemcpyAsync(dx, x, sizeof(float) * n * nc, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dy, y, sizeof(float) * n * nc, cudaMemcpyHostToDevice, s->stream);
    if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_grad_host");
    const int blocks = std::min<int>(s->part_blocks, (int)((n + TS - 1) / TS));
    if (!r) {
        mlp_grad_kernel<<<blocks, MLP_THREADS, mlp_smem_bytes(), s->stream>>>(s->w, nc, dx, dy, 0, n,
                                                                                1.f / ((float)n * nc), s->part, np);
        mlp_update_kernel<<<64, 256, 0, s->stream>>>(s->w, nc, s->master, s->m1, s->m2, s->part, blocks, np, s->grad,
                                                     0.f, 1.f, 1.f, 0);
        e = cudaGetLastError();
        if (e == cudaSuccess && grads) e = cudaMemcpyAsync(grads, s->grad, sizeof(float) * np, cudaMemcpyDeviceToHost, s->stream);
        float l = 0.f;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&l, s->grad + np, sizeof(float), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_grad_host");
        if (loss) *loss = l / ((float)n * nc);
    }
    cudaFree(dx); cudaFree(dy);
    return r;
}

int cl_eq_set_network_path(cl_eq_solver* s, int32_t path) {
    if (!s) { set_error("null argument"); return CL_ERR_ARG; }
    if (path != CL_EQ_NET_TCGEN05 && path != CL_EQ_NET_MMA_SYNC) {
        set_error("cl_eq_set_network_path: CL_EQ_NET_TCGEN05 or CL_EQ_NET_MMA_SYNC");
        return CL_ERR_ARG;
    }
    s->net_path = path;
    return CL_OK;
}

int cl_eq_predict_host(cl_eq_solver* s, const float* x, float* y, int32_t n) {
    if (!s || !x || !y || n <= 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (refuse_large(s, "cl_eq_predict_host")) return CL_ERR_ARG;
    const int nc = s->nc;
    float *dx = nullptr, *dy = nullptr;
    CL_CUDA(cudaMalloc(&dx, sizeof(float) * n * nc));
    CL_CUDA(cudaMalloc(&dy, sizeof(float) * n * nc));
    int r = CL_OK;
    cudaError_t e = cudaMemcpyAsync(dx, x, sizeof(float) * n * nc, cudaMemcpyHostToDevice, s->stream);
    if (e == cudaSuccess) r = predict_launch(s, nullptr, nullptr, dx, dy, n);
    if (e == cudaSuccess && r == CL_OK) {
        e = cudaMemcpyAsync(y, dy, sizeof(float) * n * nc, cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e == cudaSuccess) r = tc_error(s, "cl_eq_predict_host");
    }
    if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_predict_host");
    cudaFree(dx); cudaFree(dy);
    return r;
}

}  // extern "C"

namespace cl {

// standardised training arrays: Xn = (log10 T - mu_in)/sd_in, Yn = (x - log10 T - mu_out)/sd_out
__global__ void mlp_prepare_kernel(const double* T, const double* X, int64_t n, int nc, const float* norm,
                                   float* Xn, float* Yn) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * nc; i += (int64_t)gridDim.x * blockDim.x) {
        const int k = (int)(i % nc);
        const double u = log10(fmax(T[i], 1e-30));
        Xn[i] = (float)((u - norm[k]) / norm[nc + k]);
        Yn[i] = (float)((X[i] - u - norm[2 * nc + k]) / norm[3 * nc + k]);
    }
}

}  // namespace cl

extern "C" int cl_eq_train(cl_eq_solver* s, const double* d_totals, const double* d_logfree, int64_t n_pairs,
                           int32_t epochs, int32_t batch, float lr, uint64_t seed, float* final_loss) {
    if (!s || !d_totals || !d_logfree || n_pairs < TS || epochs < 1 || batch < TS) {
        set_error("cl_eq_train: bad arguments"); return CL_ERR_ARG;
    }
    if (refuse_large(s, "cl_eq_train")) return CL_ERR_ARG;
    const int nc = s->nc, np = s->n_params;
    // normalisation from a strided sample of at most 65536 pairs
    const int64_t m = std::min<int64_t>(n_pairs, 65536);
    const int64_t stride = n_pairs / m;
    std::vector<double> hT(m * nc), hX(m * nc);
    const size_t row = sizeof(double) * nc;
    CL_CUDA(cudaMemcpy2DAsync(hT.data(), row, d_totals, row * stride, row, m, cudaMemcpyDeviceToHost, s->stream));
    CL_CUDA(cudaMemcpy2DAsync(hX.data(), row, d_logfree, row * stride, row, m, cudaMemcpyDeviceToHost, s->stream));
    CL_CUDA(cudaStreamSynchronize(s->stream));
    std::vector<float> norm(4 * CL_MAX_COMP, 0.f);
    for (int k = 0; k < nc; ++k) {
        double su = 0, suu = 0, sv = 0, svv = 0;
        for (int64_t i = 0; i < m; ++i) {
            const double u = std::log10(std::max(hT[i * nc + k], 1e-30)), v = hX[i * nc + k] - u;
            su += u; suu += u * u; sv += v; svv += v * v;
        }
        const double mu = su / m, mv = sv / m;
        norm[k] = (float)mu;
        norm[nc + k] = (float)std::max(std::sqrt(std::max(suu / m - mu * mu, 0.0)), 1e-3);
        norm[2 * nc + k] = (float)mv;
        norm[3 * nc + k] = (float)std::max(std::sqrt(std::max(svv / m - mv * mv, 0.0)), 1e-3);
    }
    CL_CUDA(cudaMemcpyAsync(s->w.norm, norm.data(), sizeof(float) * norm.size(), cudaMemcpyHostToDevice, s->stream));
    float *Xn = nullptr, *Yn = nullptr;
    CL_CUDA(cudaMalloc(&Xn, sizeof(float) * n_pairs * nc));
    CL_CUDA(cudaMalloc(&Yn, sizeof(float) * n_pairs * nc));
    mlp_prepare_kernel<<<grid_for(n_pairs * nc, 256, 148 * 8), 256, 0, s->stream>>>(d_totals, d_logfree, n_pairs, nc,
                                                                                     s->w.norm, Xn, Yn);
    int r = CL_OK;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_fail(e, "mlp_prepare_kernel");
    const int64_t nb = n_pairs / batch;
    const int blocks = std::min<int>(s->part_blocks, (batch + TS - 1) / TS);
    float l = 0.f;
    std::mt19937_64 rng(seed);
    std::vector<int64_t> order(nb);
    for (int64_t i = 0; i < nb; ++i) order[i] = i;
    const double total_steps = (double)epochs * (double)nb;
    int64_t step = 0;
    for (int ep = 0; ep < epochs && !r; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        for (int64_t bi = 0; bi < nb; ++bi, ++step) {
            ++s->adam_t;
            const float b1c = 1.f - std::pow(0.9f, (float)s->adam_t), b2c = 1.f - std::pow(0.999f, (float)s->adam_t);
            // cosine decay of the learning rate over the whole run, floor 5% of lr
            const float lr_t = lr * (float)(0.05 + 0.95 * 0.5 * (1.0 + std::cos(3.141592653589793 * step / total_steps)));
            mlp_grad_kernel<<<blocks, MLP_THREADS, mlp_smem_bytes(), s->stream>>>(
                s->w, nc, Xn, Yn, order[bi] * batch, batch, 1.f / ((float)batch * nc), s->part, np);
            mlp_update_kernel<<<64, 256, 0, s->stream>>>(s->w, nc, s->master, s->m1, s->m2, s->part, blocks, np,
                                                         (bi == nb - 1) ? s->grad : nullptr, lr_t, b1c, b2c, 1);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) r = cuda_fail(e, "mlp training");
    }
    if (!r) {
        e = cudaMemcpyAsync(&l, s->grad + np, sizeof(float), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "cl_eq_train");
    }
    if (final_loss) *final_loss = l / ((float)batch * nc);
    cudaFree(Xn); cudaFree(Yn);
    if (!r) s->trained = true;
    return r;
}

// ---------------------------------------------------------------------------
// Batch speciation that allocates nothing.
//
// For callers that must not allocate device memory themselves or have the
// library do it: host code that runs under a framework's caching allocator,
// which owns the GPU's memory budget and would be bypassed by cudaMalloc, and
// code placed between the kernels of a stream-ordered sequence, where
// cudaMalloc / cudaFree would synchronise the whole device.  Such a caller
// passes its own input and output buffers; the only scratch the solve needs,
// the compacted list of voxels that fall back to the cold start, lives in the
// fixed array below, which every GPU that loads this library holds until the
// process exits.
// ---------------------------------------------------------------------------
namespace cl {

// slot 0: the fallback counter; slots kNoAllocListOffset.. : the fallback list
constexpr int64_t kNoAllocListOffset = 32;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kNoAllocListOffset + CL_EQ_NOALLOC_MAX_N];

static std::mutex g_noalloc_mu;
static unsigned long long* g_noalloc_ptr[CL_EQ_NOALLOC_MAX_DEVICES] = {};

// Device address of the scratch array on the current device.  In host code
// the symbol is only a stand-in, so the address is looked up once per device
// (with that device current) and cached.
static int noalloc_scratch(unsigned long long** out) {
    int dev = 0;
    CL_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= CL_EQ_NOALLOC_MAX_DEVICES) {
        set_error("cl_eq_solve_noalloc: device ordinal beyond the supported range");
        return CL_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        g_noalloc_ptr[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return CL_OK;
}

}  // namespace cl

extern "C" int cl_eq_solve_noalloc(const cl_eq_system* sys, const double* d_totals, const double* d_cold_species,
                                   double* d_logfree, int32_t* d_iters, uint8_t* d_status, int64_t n, int32_t start,
                                   void* stream) {
    if (!sys || sys->n_comp < 1 || sys->n_comp > 5 || sys->n_species < sys->n_comp || sys->n_species > kEqDevSpecies) {
        set_error("cl_eq_solve_noalloc: 1..5 components and n_comp <= n_species <= 16");
        return CL_ERR_ARG;
    }
    if (!d_totals || !d_logfree || n < 0) { set_error("cl_eq_solve_noalloc: null argument"); return CL_ERR_ARG; }
    if (n > CL_EQ_NOALLOC_MAX_N) {
        set_error("cl_eq_solve_noalloc: n exceeds CL_EQ_NOALLOC_MAX_N (1048576); split the batch");
        return CL_ERR_ARG;
    }
    if (start != CL_EQ_START_COLD && start != CL_EQ_START_GIVEN) {
        set_error("cl_eq_solve_noalloc: start must be CL_EQ_START_COLD or CL_EQ_START_GIVEN");
        return CL_ERR_ARG;
    }
    if (start == CL_EQ_START_COLD && !d_cold_species) {
        set_error("cl_eq_solve_noalloc: the cold start needs the species vectors");
        return CL_ERR_ARG;
    }
    if (n == 0) return CL_OK;
    unsigned long long* scratch = nullptr;
    int r = noalloc_scratch(&scratch);
    if (r) return r;
    cudaStream_t st = (cudaStream_t)stream;
    EqDev e;
    eqdev_from_system(*sys, e);
    const bool fallback = (start == CL_EQ_START_GIVEN) && d_cold_species != nullptr;
    unsigned long long* count = scratch;
    int64_t* list = reinterpret_cast<int64_t*>(scratch + kNoAllocListOffset);
    if (fallback) CL_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
    const int limit = (start == CL_EQ_START_COLD) ? sys->max_iter : sys->warm_iter;
    const int blocks = grid_for(n, 128, 148 * 16);
#define CL_NA_FIRST(NCV) newton_first_kernel<NCV><<<blocks, 128, 0, st>>>(e, d_totals, d_cold_species, d_logfree, d_iters, d_status, n, start, limit, sys->tol, fallback ? list : nullptr, count)
#define CL_NA_FB(NCV) newton_fallback_kernel<NCV><<<blocks, 128, 0, st>>>(e, d_totals, d_cold_species, d_logfree, d_iters, d_status, list, count, sys->max_iter, sys->tol)
    switch (sys->n_comp) {
        case 1: CL_NA_FIRST(1); if (fallback) CL_NA_FB(1); break;
        case 2: CL_NA_FIRST(2); if (fallback) CL_NA_FB(2); break;
        case 3: CL_NA_FIRST(3); if (fallback) CL_NA_FB(3); break;
        case 4: CL_NA_FIRST(4); if (fallback) CL_NA_FB(4); break;
        default: CL_NA_FIRST(5); if (fallback) CL_NA_FB(5); break;
    }
#undef CL_NA_FIRST
#undef CL_NA_FB
    CL_LAUNCH_CHECK("cl_eq_solve_noalloc");
    return CL_OK;
}

namespace cl {
__global__ void exp10_check_kernel(const double* x, double* y, int64_t n, int which) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = which ? exp10(x[i]) : cl_exp10(x[i]);
}
}  // namespace cl

extern "C" int cl_math_exp10(const double* x, double* y, int64_t n, int32_t which) {
    if (!x || !y || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (n == 0) return CL_OK;
    double* d = nullptr;
    CL_CUDA(cudaMalloc(&d, sizeof(double) * 2 * n));
    cudaError_t e = cudaMemcpy(d, x, sizeof(double) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        cl::exp10_check_kernel<<<cl::grid_for(n, 256, 148 * 8), 256>>>(d, d + n, n, which);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? CL_OK : cl::cuda_fail(e, "cl_math_exp10");
}
