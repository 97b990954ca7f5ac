// surrogate.cu -- batched per-voxel inference of the surrogate rate network.
//
// The reference evaluates its exported feed-forward network one voxel at a
// time with std::vector mat-vec loops (defineSurrogateModel,
// surrogateModel.hh:252-501): mapminmax input scaling xs = (x - offset)*gain +
// ymin, tansig hidden layers (tansig(n) = 2/(1+exp(-2n)) - 1 = tanh n), a
// linear output layer, and the reverse mapminmax on the output.
//
// CL_SRG_TENSOR: one warp carries 16 voxels through every layer with BF16
//   m16n8k16 tensor-core MMAs (FP32 accumulate); weights are staged once per
//   block in shared memory, padded to K multiples of 16 and N multiples of 8.
// CL_SRG_TCGEN05: 128 voxels per CTA through tcgen05.mma (M = 128, K and N
//   padded to 16 and 32 columns), FP32 accumulators in tensor memory.
// CL_SRG_FP32: the FP32 CUDA-core reference kernel, one voxel per thread.
#include "internal.h"
#include "mma.cuh"
#include "umma.cuh"

namespace cl {

constexpr int SW = CL_SRG_MAX_WIDTH;     // 32
constexpr int SP = SW + 8;               // activation / weight row pitch (bf16)
constexpr int SRG_WARPS = 8;

struct SrgDev {
    int L;
    int w[CL_SRG_MAX_LAYERS + 1];
    float xo[SW], xg[SW], xymin, yo[SW], yg[SW], yymin, xlo[SW], xhi[SW];
    int poff[CL_SRG_MAX_LAYERS];   // offset of layer l's weights in the packed FP32 array
};

__host__ __device__ inline int pad16(int v) { return (v + 15) / 16 * 16; }
__host__ __device__ inline int pad8(int v) { return (v + 7) / 8 * 8; }

// tensor-core inference: smem = weights [L][SW][SP] bf16 + biases [L][SW] f32 +
// per-warp activation ping-pong buffers [warps][2][16][SP] bf16
__global__ void __launch_bounds__(SRG_WARPS * 32) srg_tensor_kernel(SrgDev d, const float* params, const float* x,
                                                                     float* y, int64_t n) {
    extern __shared__ __align__(16) unsigned char sm[];
    __nv_bfloat16* W = reinterpret_cast<__nv_bfloat16*>(sm);
    float* B = reinterpret_cast<float*>(sm + sizeof(__nv_bfloat16) * CL_SRG_MAX_LAYERS * SW * SP);
    __nv_bfloat16* act = reinterpret_cast<__nv_bfloat16*>(B + CL_SRG_MAX_LAYERS * SW);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    // stage weights W[l][o][i] (zero padded) and biases
    for (int l = 0; l < d.L; ++l) {
        const int wi = d.w[l], wo = d.w[l + 1];
        const float* p = params + d.poff[l];
        for (int e = threadIdx.x; e < SW * SP; e += blockDim.x) {
            const int o = e / SP, i = e - o * SP;
            const float v = (o < wo && i < wi) ? p[o * wi + i] : 0.f;
            W[(l * SW + o) * SP + i] = __float2bfloat16_rn(v);
        }
        for (int o = threadIdx.x; o < SW; o += blockDim.x) B[l * SW + o] = (o < wo) ? p[wo * wi + o] : 0.f;
    }
    __syncthreads();
    __nv_bfloat16* a0 = act + warp * 2 * 16 * SP;
    __nv_bfloat16* a1 = a0 + 16 * SP;
    const int64_t ntiles = (n + 15) / 16;
    const int win = d.w[0], wout = d.w[d.L];
    for (int64_t tile = (int64_t)blockIdx.x * SRG_WARPS + warp; tile < ntiles; tile += (int64_t)gridDim.x * SRG_WARPS) {
        const int64_t s0 = tile * 16;
        // input: clamp, mapminmax, bf16; zero the padding columns
        for (int e = lane; e < 16 * SP; e += 32) {
            const int m = e / SP, i = e - m * SP;
            float v = 0.f;
            if (i < win && s0 + m < n) {
                float xv = x[(s0 + m) * win + i];
                xv = fminf(fmaxf(xv, d.xlo[i]), d.xhi[i]);
                v = (xv - d.xo[i]) * d.xg[i] + d.xymin;
            }
            a0[e] = __float2bfloat16_rn(v);
        }
        __syncwarp();
        __nv_bfloat16* cur = a0;
        __nv_bfloat16* nxt = a1;
        for (int l = 0; l < d.L; ++l) {
            const int K = pad16(d.w[l]), N = pad8(d.w[l + 1]);
            const bool last = (l == d.L - 1);
            for (int n0 = 0; n0 < N; n0 += 8) {
                float acc[4] = {0.f, 0.f, 0.f, 0.f};
                warp_tile(acc, cur, SP, 0, W + l * SW * SP, SP, n0, K);
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    const int m = g + (r >> 1) * 8, o = n0 + 2 * t + (r & 1);
                    float v = acc[r] + B[l * SW + o];
                    if (!last) {
                        v = tanhf(v);
                        nxt[m * SP + o] = __float2bfloat16_rn(o < d.w[l + 1] ? v : 0.f);
                    } else if (o < wout && s0 + m < n) {
                        y[(s0 + m) * wout + o] = (v - d.yymin) / d.yg[o] + d.yo[o];
                    }
                }
            }
            if (!last) {
                // zero the K padding of the next layer's input beyond N
                const int Kn = pad16(d.w[l + 1]);
                for (int e = lane; e < 16 * (Kn - N); e += 32) {
                    const int m = e / (Kn - N), i = N + e % (Kn - N);
                    nxt[m * SP + i] = __float2bfloat16_rn(0.f);
                }
            }
            __syncwarp();
            __nv_bfloat16* tmp = cur; cur = nxt; nxt = tmp;
        }
    }
}

// The same inference on the fifth-generation tensor core: one voxel per
// thread and TMEM lane, 128 per CTA; per layer one thread issues K/16 MMAs
// (K = pad16 of the layer's input width, N = pad16 of its output width, both
// at most 32) on the activation tile and the layer's weights, held in shared
// memory as K-major 8x8 core matrices (umma.cuh); the epilogue reads the
// thread's row from TMEM, adds the bias, applies tansig and writes the next
// layer's BF16 operand (the output layer: the reverse mapminmax).  Every wait
// on the MMAs is bounded; a timeout sets g_srg_tc_err and the CTA stops.
__device__ unsigned int g_srg_tc_err;
constexpr int SRG_TC = 128;

struct SrgSmemTc {
    alignas(128) unsigned char act[SRG_TC * SW * 2];                 // [128][32]
    alignas(128) unsigned char W[CL_SRG_MAX_LAYERS][SW * SW * 2];    // [32 out][32 in] per layer
    float B[CL_SRG_MAX_LAYERS][SW];
    alignas(8) unsigned long long bar;
    uint32_t tmem;
};

__global__ void __launch_bounds__(SRG_TC) srg_tc_kernel(SrgDev d, const float* params, const float* x, float* y,
                                                        int64_t n) {
    extern __shared__ __align__(16) unsigned char sm[];
    SrgSmemTc& s = *reinterpret_cast<SrgSmemTc*>(sm);
    const int tid = threadIdx.x, warp = tid >> 5;
    for (int l = 0; l < d.L; ++l) {
        const int wi = d.w[l], wo = d.w[l + 1];
        const float* p = params + d.poff[l];
        for (int e = tid; e < SW * SW; e += SRG_TC) {
            const int o = e / SW, i = e - o * SW;
            const float v = (o < wo && i < wi) ? p[o * wi + i] : 0.f;
            *reinterpret_cast<__nv_bfloat16*>(s.W[l] + umma_off(o, i, SW / 8)) = __float2bfloat16_rn(v);
        }
        for (int o = tid; o < SW; o += SRG_TC) s.B[l][o] = (o < wo) ? p[wo * wi + o] : 0.f;
    }
    const uint32_t bar = smem_u32(&s.bar);
    if (tid == 0) mbar_init(bar, 1);
    if (warp == 0) tmem_alloc(smem_u32(&s.tmem), 32);
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem, lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t aAct = smem_u32(s.act);
    constexpr int kLimit = 1 << 20;
    const int win = d.w[0], wout = d.w[d.L];
    uint32_t phase = 0;
    bool ok = true;
    const int64_t ntiles = (n + SRG_TC - 1) / SRG_TC;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int64_t s0 = tile * SRG_TC;
        const int m = tid;
        const bool valid = s0 + m < n;
        // input: clamp, mapminmax, BF16, zero beyond the input width
        for (int c = 0; c < SW / 8; ++c) {
            uint32_t wv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float v2[2];
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int i = 8 * c + 2 * j + h;
                    float v = 0.f;
                    if (valid && i < win) {
                        float xv = x[(s0 + m) * win + i];
                        xv = fminf(fmaxf(xv, d.xlo[i]), d.xhi[i]);
                        v = (xv - d.xo[i]) * d.xg[i] + d.xymin;
                    }
                    v2[h] = v;
                }
                wv[j] = pack_bf16(v2[0], v2[1]);
            }
            *reinterpret_cast<uint4*>(s.act + umma_off(m, 8 * c, SW / 8)) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
        }
        for (int l = 0; l < d.L; ++l) {
            const int K = pad16(d.w[l]), N = pad16(d.w[l + 1]);
            const bool last = (l == d.L - 1);
            fence_async_smem();
            tc_fence_before();
            __syncthreads();
            tc_fence_after();
            if (tid == 0) {
                const uint32_t aW = smem_u32(s.W[l]);
                for (int kb = 0; kb < K / 16; ++kb)
                    umma_bf16(tmem, umma_desc(aAct, kb, SW / 8), umma_desc(aW, kb, SW / 8), umma_idesc_bf16(N), kb > 0);
                umma_commit(bar);
            }
            if (!__syncthreads_and(mbar_wait(bar, phase & 1u, kLimit))) { ok = false; break; }
            ++phase;
            tc_fence_after();
            for (int c = 0; c < N / 16; ++c) {
                float acc[16];
                tmem_ld16(lane_addr + (uint32_t)(16 * c), acc);
                if (last) {
                    if (valid)
                        for (int j = 0; j < 16; ++j) {
                            const int o = 16 * c + j;
                            if (o < wout) y[(s0 + m) * wout + o] = (acc[j] + s.B[l][o] - d.yymin) / d.yg[o] + d.yo[o];
                        }
                } else {
                    uint32_t wv[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j) {
                        const int o = 16 * c + 2 * j;
                        const float v0 = o < d.w[l + 1] ? tanhf(acc[2 * j] + s.B[l][o]) : 0.f;
                        const float v1 = o + 1 < d.w[l + 1] ? tanhf(acc[2 * j + 1] + s.B[l][o + 1]) : 0.f;
                        wv[j] = pack_bf16(v0, v1);
                    }
                    *reinterpret_cast<uint4*>(s.act + umma_off(m, 16 * c, SW / 8)) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
                    *reinterpret_cast<uint4*>(s.act + umma_off(m, 16 * c + 8, SW / 8)) = make_uint4(wv[4], wv[5], wv[6], wv[7]);
                }
            }
            if (!last && N < SW) {
                // columns beyond this layer's output: zero
                const uint4 z = make_uint4(0u, 0u, 0u, 0u);
                for (int c = N / 8; c < SW / 8; ++c) *reinterpret_cast<uint4*>(s.act + umma_off(m, 8 * c, SW / 8)) = z;
            }
        }
    }
    if (!ok) {
        mbar_wait(bar, phase & 1u, kLimit);
        if (tid == 0) atomicOr(&g_srg_tc_err, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(tmem, 32);
}

// FP32 CUDA-core reference: one voxel per thread, weights in shared memory
__global__ void srg_fp32_kernel(SrgDev d, const float* params, int n_params, const float* x, float* y, int64_t n) {
    extern __shared__ __align__(16) unsigned char sm[];
    float* P = reinterpret_cast<float*>(sm);
    for (int i = threadIdx.x; i < n_params; i += blockDim.x) P[i] = params[i];
    __syncthreads();
    const int win = d.w[0], wout = d.w[d.L];
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
        float a[SW], b[SW];
        for (int i = 0; i < win; ++i) {
            float xv = fminf(fmaxf(x[k * win + i], d.xlo[i]), d.xhi[i]);
            a[i] = (xv - d.xo[i]) * d.xg[i] + d.xymin;
        }
        for (int l = 0; l < d.L; ++l) {
            const int wi = d.w[l], wo = d.w[l + 1];
            const float* Wl = P + d.poff[l];
            for (int o = 0; o < wo; ++o) {
                float s = Wl[wo * wi + o];
                for (int i = 0; i < wi; ++i) s = fmaf(Wl[o * wi + i], a[i], s);
                b[o] = (l < d.L - 1) ? tanhf(s) : s;
            }
            for (int o = 0; o < wo; ++o) a[o] = b[o];
        }
        for (int o = 0; o < wout; ++o) y[k * wout + o] = (a[o] - d.yymin) / d.yg[o] + d.yo[o];
    }
}

static int srg_prepare(const cl_surrogate_net* net, SrgDev& d, int& n_params) {
    if (!net || net->n_layers < 1 || net->n_layers > CL_SRG_MAX_LAYERS) { set_error("surrogate: 1..5 layers"); return CL_ERR_ARG; }
    d.L = net->n_layers;
    int off = 0;
    for (int l = 0; l <= d.L; ++l) {
        d.w[l] = net->widths[l];
        if (d.w[l] < 1 || d.w[l] > SW) { set_error("surrogate: widths must be 1..32"); return CL_ERR_ARG; }
    }
    for (int l = 0; l < d.L; ++l) { d.poff[l] = off; off += d.w[l + 1] * d.w[l] + d.w[l + 1]; }
    if (off > 4096) { set_error("surrogate: too many parameters"); return CL_ERR_ARG; }
    n_params = off;
    for (int i = 0; i < SW; ++i) {
        d.xo[i] = (float)net->x_offset[i]; d.xg[i] = (float)net->x_gain[i];
        d.yo[i] = (float)net->y_offset[i]; d.yg[i] = (float)net->y_gain[i];
        d.xlo[i] = (float)net->x_lo[i]; d.xhi[i] = (float)net->x_hi[i];
    }
    d.xymin = (float)net->x_ymin; d.yymin = (float)net->y_ymin;
    return CL_OK;
}

}  // namespace cl

using namespace cl;

extern "C" int cl_surrogate_batch_device(const cl_surrogate_net* net, const float* d_x, float* d_y, int64_t n,
                                         int32_t mode, void* stream) {
    SrgDev d;
    int np = 0;
    int r = srg_prepare(net, d, np);
    if (r) return r;
    if (!d_x || !d_y || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (n == 0) return CL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    float* dp = nullptr;
    CL_CUDA(cudaMallocAsync(&dp, sizeof(float) * np, st));
    float hp[4096];
    for (int i = 0; i < np; ++i) hp[i] = (float)net->params[i];
    CL_CUDA(cudaMemcpyAsync(dp, hp, sizeof(float) * np, cudaMemcpyHostToDevice, st));
    if (mode == CL_SRG_TENSOR) {
        const size_t smem = sizeof(__nv_bfloat16) * CL_SRG_MAX_LAYERS * SW * SP + sizeof(float) * CL_SRG_MAX_LAYERS * SW +
                            sizeof(__nv_bfloat16) * SRG_WARPS * 2 * 16 * SP;
        CL_CUDA(cudaFuncSetAttribute(srg_tensor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int64_t tiles = (n + 15) / 16;
        const int blocks = grid_for(tiles, SRG_WARPS, 148 * 4);
        srg_tensor_kernel<<<blocks, SRG_WARPS * 32, smem, st>>>(d, dp, d_x, d_y, n);
    } else if (mode == CL_SRG_TCGEN05) {
        CL_CUDA(cudaFuncSetAttribute(srg_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(SrgSmemTc)));
        srg_tc_kernel<<<grid_for((n + SRG_TC - 1) / SRG_TC, 1, 148 * 4), SRG_TC, sizeof(SrgSmemTc), st>>>(d, dp, d_x,
                                                                                                          d_y, n);
    } else {
        srg_fp32_kernel<<<grid_for(n, 256, 148 * 8), 256, sizeof(float) * np, st>>>(d, dp, np, d_x, d_y, n);
    }
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(dp, st);
    if (e != cudaSuccess) return cuda_fail(e, "surrogate kernel");
    return CL_OK;
}

extern "C" int cl_surrogate_batch_host(const cl_surrogate_net* net, const float* x, float* y, int64_t n, int32_t mode) {
    if (!net || !x || !y || n < 0) { set_error("null argument"); return CL_ERR_ARG; }
    if (n == 0) return CL_OK;
    const int win = net->widths[0], wout = net->widths[net->n_layers];
    float *dx = nullptr, *dy = nullptr;
    CL_CUDA(cudaMalloc(&dx, sizeof(float) * n * win));
    CL_CUDA(cudaMalloc(&dy, sizeof(float) * n * wout));
    int r = CL_OK;
    cudaError_t e = cudaMemcpy(dx, x, sizeof(float) * n * win, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) r = cuda_fail(e, "copy");
    if (!r) r = cl_surrogate_batch_device(net, dx, dy, n, mode, nullptr);
    if (!r) {
        e = cudaMemcpy(y, dy, sizeof(float) * n * wout, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) r = cuda_fail(e, "copy");
    }
    if (!r && mode == CL_SRG_TCGEN05) {
        unsigned int v = 0;
        e = cudaMemcpyFromSymbol(&v, g_srg_tc_err, sizeof(v));
        if (e == cudaSuccess && v) {
            const unsigned int z = 0;
            cudaMemcpyToSymbol(g_srg_tc_err, &z, sizeof(z));
            set_error("cl_surrogate_batch_host: the tensor-core inference timed out waiting for its MMAs");
            r = CL_ERR_CUDA;
        } else if (e != cudaSuccess) {
            r = cuda_fail(e, "copy");
        }
    }
    cudaFree(dx); cudaFree(dy);
    return r;
}
