// ade.cu -- transport-step dispatch, initialisation and field access.
// The fused kernels themselves live in ade_kernels.cuh.
#include "ade_kernels.cuh"

namespace cl {

int ade_step(Ctx* c) {
    if (c->chem > 0 && c->chem_on) return ade_step_fast(c);
    const int nc = c->ap.do_eq ? c->cfg.eq.n_comp : 0;
    switch (nc) {
        case 0: return ade_step_nc0(c);
        case 1: return ade_step_nc1(c);
        case 2: return ade_step_nc2(c);
        case 3: return ade_step_nc3(c);
        case 4: return ade_step_nc4(c);
        case 5: return ade_step_nc5(c);
        default: set_error("equilibrium in the transport step supports 1..5 components");
                 return CL_ERR_ARG;
    }
}

// the immobile inventories and boundary densities; the populations of the
// stored sites get t_i * c0 from store_update
__global__ void ade_init_kernel(Geo g, int n_mob, AdeParams p, const double* c0, double* imm, float* rho_adj) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        for (int s = 0; s < p.S; ++s)
            if (p.mob_slot[s] < 0) imm[(int64_t)s * g.N + n] = c0[s];
        if (n < g.plane)
            for (int m = 0; m < n_mob; ++m) {
                const float c = (float)c0[p.mob_index[m]];
                rho_adj[((int64_t)m * 2 + 0) * g.plane + n] = c;
                rho_adj[((int64_t)m * 2 + 1) * g.plane + n] = c;
            }
    }
}

int ade_init(Ctx* c) {
    // storage from scratch: every slot holds its initial value again
    if (c->d_sidx) CL_CUDA(cudaMemsetAsync(c->d_sidx, 0xff, sizeof(int32_t) * c->geo.N, c->stream));
    c->n_stored = 0;
    int r = store_update(c, 0);
    if (r) return r;
    double* d_c0 = c->d_scratch;   // S doubles
    CL_CUDA(cudaMemcpyAsync(d_c0, c->cfg.c0, sizeof(double) * c->ap.S, cudaMemcpyHostToDevice, c->stream));
    ade_init_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(
        c->geo, c->ap.n_mob, c->ap, d_c0, c->d_imm, c->d_rho_adj);
    CL_LAUNCH_CHECK("ade_init_kernel");
    c->ade_parity = 0;
    return CL_OK;
}

// computeDensity of every site.  A dynamic cell on an x face answers with its
// prescribed density: the Dirichlet value, or on a zero-gradient face the
// current density of the neighbour plane (what FlatAdiabaticBoundaryFunctional3D
// copies after each stream).
template <int PARITY>
__device__ __forceinline__ double site_density(Geo g, const float* pm, const int32_t* sidx, float c0, int64_t n) {
    int x, y, z;
    decode(g, n, x, y, z);
    float f[7];
    gather7_any<PARITY>(pm, (uint32_t)g.N, sidx, g, x, y, z, (uint32_t)n, c0, f);
    double r = 0.0;
#pragma unroll
    for (int i = 0; i < 7; ++i) r += f[i];
    return r;
}

template <int PARITY>
__global__ void ade_density_kernel(Geo g, const float* pm, const int32_t* sidx, float c0, const uint8_t* cls,
                                   int lneu, int rneu, double lval, double rval, double* out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        const uint8_t dyn = cls[n] & 3;
        const bool dynamic = dyn == FLUID || dyn == BIO;
        if (dynamic && n < g.plane) out[n] = lneu ? site_density<PARITY>(g, pm, sidx, c0, n + g.plane) : lval;
        else if (dynamic && n >= g.N - g.plane)
            out[n] = rneu ? site_density<PARITY>(g, pm, sidx, c0, n - g.plane) : rval;
        else out[n] = site_density<PARITY>(g, pm, sidx, c0, n);
    }
}

int ade_density(Ctx* c, int s, double* d_out) {
    const int slot = c->ap.mob_slot[s];
    if (slot < 0) {
        CL_CUDA(cudaMemcpyAsync(d_out, c->d_imm + (int64_t)s * c->geo.N, sizeof(double) * c->geo.N,
                                cudaMemcpyDeviceToDevice, c->stream));
        return CL_OK;
    }
    const float* pm = c->d_g + (int64_t)slot * 7 * c->geo.N;
    const int blocks = grid_for(c->geo.N, 256, 148 * 16);
    const int ln = c->ap.left_neu[slot], rn = c->ap.right_neu[slot];
    const double lv = c->cfg.left_value[s], rv = c->cfg.right_value[s];
    const float c0 = (float)c->cfg.c0[s];
    if (c->ade_parity == 0)
        ade_density_kernel<0><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, c0, c->d_ade_cls, ln, rn, lv, rv, d_out);
    else
        ade_density_kernel<1><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, c0, c->d_ade_cls, ln, rn, lv, rv, d_out);
    CL_LAUNCH_CHECK("ade_density_kernel");
    return CL_OK;
}

template <int PARITY>
__global__ void ade_io_kernel(Geo g, const float* pm, const int32_t* sidx, float c0, float* nat) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        int x, y, z;
        decode(g, n, x, y, z);
        float f[7];
        gather7_any<PARITY>(pm, (uint32_t)g.N, sidx, g, x, y, z, (uint32_t)n, c0, f);
#pragma unroll
        for (int i = 0; i < 7; ++i) nat[i * g.N + n] = f[i];
    }
}

int ade_population_io(Ctx* c, int slot, float* d_nat) {
    const float* pm = c->d_g + (int64_t)slot * 7 * c->geo.N;
    const int blocks = grid_for(c->geo.N, 256, 148 * 16);
    const float c0 = (float)c->cfg.c0[c->ap.mob_index[slot]];
    if (c->ade_parity == 0) ade_io_kernel<0><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, c0, d_nat);
    else ade_io_kernel<1><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, c0, d_nat);
    CL_LAUNCH_CHECK("ade_io_kernel");
    return CL_OK;
}

}  // namespace cl
