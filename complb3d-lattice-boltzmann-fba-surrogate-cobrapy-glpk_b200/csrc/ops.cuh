// ops.cuh -- the transport step taken apart: collide, the reaction
// processors one at a time, stream.  These kernels back the per-operator
// entry points (cl_op_*), which keep the reference's call structure
// (src/complab.cpp:1252-1374, 1849-1857: collide, run_kinetics /
// run_surrogate3D + update_rxnLattices, the abiotic processors +
// update_abiotic_rxnLattices, run_equilibrium_biotic, stream).  The fused
// step (cl_step) does the same work in one or two launches per step; these
// take one launch per processor and write the populations back to the slots
// they were read from between the calls.
#pragma once
#include "ade_kernels.cuh"

namespace cl {

// the slot population i of a site is read from at this parity (gather7's address)
template <int PARITY>
__device__ __forceinline__ uint32_t slot7(uint32_t N, const SSite& st, int i) {
    if (i == 0) return st.s;
    if (PARITY == 0 || !st.inx(-c7x(i))) return (uint32_t)i * N + st.s;
    return (uint32_t)opp7(i) * N + st.nb[opp7(i) - 1];
}

// the reaction processors selected by ops on the current populations of every
// reactive site; each mobile solute's total increment t_i * dC goes back into
// the slots the site's populations occupy
template <int NC, int PARITY, int SOLVER>
__global__ void __launch_bounds__(kReactBlock) ade_ops_kernel(const __grid_constant__ AdeK k,
                                                              const uint32_t* __restrict__ list, int64_t count,
                                                              int ops) {
    extern __shared__ double sm[];
    const int t = threadIdx.x;
    const AdeParams& p = k.p;
    const int Mw = p.M > 0 ? p.M : 1;
    double* Cur = sm;
    double* App = Cur + p.S * kReactBlock;
    double* Rw = App + p.S * kReactBlock;
    double* Bw = Rw + p.S * kReactBlock;
    double* BRw = Bw + Mw * kReactBlock;
    const int64_t N = k.g.N;
    const uint32_t N32 = (uint32_t)N;
    unsigned long long nonconv = 0;
    double* cCur = Cur + t;
    double* cApp = App + t;
    for (int64_t r = (int64_t)blockIdx.x * kReactBlock + t; r < count; r += (int64_t)gridDim.x * kReactBlock) {
        const uint32_t n = list[r];
        const uint8_t cls = k.cls[n];
        if (!(cls & F_REACTIVE)) continue;
        int x, y, z;
        decode(k.g, n, x, y, z);
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) { atomicAdd(&k.counters[1], 1ull); continue; }
        for (int s = 0; s < p.S; ++s) cApp[s * kReactBlock] = 0.0;
        for (int m = 0; m < p.n_mob; ++m) {
            float f[7];
            gather7<PARITY>(k.pop + (int64_t)m * 7 * N, N32, st, f);
            float rr = 0.f;
#pragma unroll
            for (int i = 0; i < 7; ++i) rr += f[i];
            cCur[p.mob_index[m] * kReactBlock] = (double)rr;
        }
        for (int s = 0; s < p.S; ++s)
            if (p.mob_slot[s] < 0) cCur[s * kReactBlock] = k.imm[(int64_t)s * N + n];
        nonconv += reaction_chain<NC, SOLVER>(k, n, st.s, x, y, z, cls, cCur, cApp, kReactBlock, Rw + t, Bw + t,
                                              BRw + t, kReactBlock, ops);
        for (int s = 0; s < p.S; ++s)
            if (p.mob_slot[s] < 0 && cApp[s * kReactBlock] != 0.0) k.imm[(int64_t)s * N + n] += cApp[s * kReactBlock];
        for (int m = 0; m < p.n_mob; ++m) {
            const float d = (float)cApp[p.mob_index[m] * kReactBlock];
            if (d == 0.f) continue;
            float* pm = k.pop + (int64_t)m * 7 * N;
#pragma unroll
            for (int i = 0; i < 7; ++i) pm[slot7<PARITY>(N32, st, i)] += t7(i) * d;
        }
    }
    for (int o = 16; o > 0; o >>= 1) nonconv += __shfl_down_sync(0xffffffffu, nonconv, o);
    if ((t & 31) == 0 && nonconv) atomicAdd(&k.counters[0], nonconv);
}

template <int NC>
inline int launch_ops(Ctx* c, const AdeK& k, int ops) {
    if (c->n_live <= 0) return CL_OK;
    const int S = c->ap.S, M = c->ap.M > 0 ? c->ap.M : 1;
    const size_t smem = (size_t)(3 * S + 2 * M) * kReactBlock * sizeof(double);
    const int blocks = grid_for(c->n_live, kReactBlock, 148 * 8);
    const bool pcf = NC > 0 && k.e.solver == CL_EQ_SOLVER_PCF;
    constexpr int PCF = NC > 0 ? CL_EQ_SOLVER_PCF : CL_EQ_SOLVER_NEWTON;
    auto go = [&](auto kern) -> int {
        CL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<blocks, kReactBlock, smem, c->stream>>>(k, c->d_live, c->n_live, ops);
        CL_LAUNCH_CHECK("ade_ops_kernel");
        c->launches += 1;
        return CL_OK;
    };
    if (c->ade_parity == 0)
        return pcf ? go(ade_ops_kernel<NC, 0, PCF>) : go(ade_ops_kernel<NC, 0, CL_EQ_SOLVER_NEWTON>);
    return pcf ? go(ade_ops_kernel<NC, 1, PCF>) : go(ade_ops_kernel<NC, 1, CL_EQ_SOLVER_NEWTON>);
}

// one translation unit per component count instantiates these
int ade_ops_nc0(Ctx* c, const AdeK& k, int ops); int ade_ops_nc1(Ctx* c, const AdeK& k, int ops);
int ade_ops_nc2(Ctx* c, const AdeK& k, int ops); int ade_ops_nc3(Ctx* c, const AdeK& k, int ops);
int ade_ops_nc4(Ctx* c, const AdeK& k, int ops); int ade_ops_nc5(Ctx* c, const AdeK& k, int ops);

}  // namespace cl
