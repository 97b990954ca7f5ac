// ade.cu -- transport-step dispatch, initialisation and field access.
// The fused kernels themselves live in ade_kernels.cuh.
#include "ade_kernels.cuh"

namespace cl {

int ade_step(Ctx* c) {
    if (c->chem > 0 && c->chem_on && chem_ready(c)) return ade_step_fast(c);
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

// Where population i of site n lives at this parity (the address gather7_any
// reads): slot i of n itself, or in the odd parity, when the upstream
// neighbour n - c_i is inside the x range, slot opp(i) of that neighbour.
template <int PARITY>
__device__ __forceinline__ void nat_slot(const Geo& g, int x, int y, int z, uint32_t n, int i, uint32_t& owner,
                                         int& idx) {
    owner = n;
    idx = i;
    if (PARITY == 1 && i > 0) {
        const Site st = make_site(g, x, y, z, n);
        if (st.inx(-c7x(i))) { owner = st.at(-c7x(i), -c7y(i), -c7z(i)); idx = opp7(i); }
    }
}

// the sites that must hold storage for natural-order populations: the owner
// of every slot whose value is not the initial t_i c0 an unstored slot reads
template <int PARITY>
__global__ void ade_nat_need_kernel(Geo g, const float* nat, float c0, uint8_t* need) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        int x, y, z;
        decode(g, n, x, y, z);
        for (int i = 0; i < 7; ++i) {
            uint32_t owner;
            int idx;
            nat_slot<PARITY>(g, x, y, z, (uint32_t)n, i, owner, idx);
            if (nat[i * g.N + n] != t7(idx) * c0) need[owner] = 1;
        }
    }
}

template <int PARITY>
__global__ void ade_nat_write_kernel(Geo g, float* pm, const int32_t* sidx, const float* nat) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        int x, y, z;
        decode(g, n, x, y, z);
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            uint32_t owner;
            int idx;
            nat_slot<PARITY>(g, x, y, z, (uint32_t)n, i, owner, idx);
            const int32_t s = sidx[owner];
            if (s >= 0) pm[idx * g.N + (uint32_t)s] = nat[i * g.N + n];
        }
    }
}

// natural-order populations of a mobile solute into the storage at this
// parity; sites whose slots receive anything but their initial value are
// stored first, so a checkpoint of a compact run restores compactly
int ade_population_set(Ctx* c, int slot, const float* d_nat) {
    const int64_t N = c->geo.N;
    const int blocks = grid_for(N, 256, 148 * 16);
    const float c0 = (float)c->cfg.c0[c->ap.mob_index[slot]];
    uint8_t* need = nullptr;
    CL_CUDA(cudaMalloc(&need, (size_t)N));
    cudaError_t e = cudaMemsetAsync(need, 0, (size_t)N, c->stream);
    if (e == cudaSuccess) {
        if (c->ade_parity == 0) ade_nat_need_kernel<0><<<blocks, 256, 0, c->stream>>>(c->geo, d_nat, c0, need);
        else ade_nat_need_kernel<1><<<blocks, 256, 0, c->stream>>>(c->geo, d_nat, c0, need);
        e = cudaGetLastError();
    }
    int r = e == cudaSuccess ? store_update(c, 0, need) : cuda_fail(e, "ade_population_set");
    if (!r) {
        float* pm = c->d_g + (int64_t)slot * 7 * N;
        if (c->ade_parity == 0) ade_nat_write_kernel<0><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, d_nat);
        else ade_nat_write_kernel<1><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, d_nat);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "ade_nat_write_kernel");
    }
    cudaFree(need);
    return r;
}

// the Newton warm starts (FP32 by storage index) <-> FP64 in site order;
// sites without storage read NaN (no previous solution)
__global__ void eq_start_get_kernel(int64_t N, const int32_t* sidx, const float* col, double* out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        const int32_t s = sidx[n];
        out[n] = s >= 0 ? (double)col[s] : __longlong_as_double(0x7ff8000000000000ll);
    }
}
__global__ void eq_start_set_kernel(int64_t N, const int32_t* sidx, float* col, const double* in) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N; n += stride) {
        const int32_t s = sidx[n];
        if (s >= 0) col[s] = (float)in[n];
    }
}

int eq_start_io(Ctx* c, int j, double* d_nat, int to_natural) {
    const int nc = c->cfg.eq.n_comp;
    if (!c->d_eq_x || j < 0 || j >= 2 * nc) { set_error("no warm starts in this context, or index out of range"); return CL_ERR_ARG; }
    // (a read brings the storage up to date first; a write finds it so)
    if (to_natural && c->store_dirty) { int r = store_update(c, 0); if (r) return r; }
    const int64_t N = c->geo.N;
    float* col = (j < nc ? c->d_eq_x : c->d_eq_xp) + (int64_t)(j % nc) * N;
    const int blocks = grid_for(N, 256, 148 * 16);
    if (to_natural) eq_start_get_kernel<<<blocks, 256, 0, c->stream>>>(N, c->d_sidx, col, d_nat);
    else eq_start_set_kernel<<<blocks, 256, 0, c->stream>>>(N, c->d_sidx, col, d_nat);
    CL_LAUNCH_CHECK("eq_start_io");
    return CL_OK;
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
