// ops.cu -- the per-operator entry points: the transport step as collide,
// the reaction processors one by one, and stream (ops.cuh), in the order the
// reference calls its processors (src/complab.cpp:1252-1374, 1849-1857).
#include "ops.cuh"

namespace cl {

// AdvectionDiffusionBGKdynamics collide in place: each site's populations go
// back to the slots they were read from; bounce-back sites swap, NoDynamics
// sites keep theirs.  The density next to each x face is recorded for the
// zero-gradient faces, as the fused step records it.
template <int PARITY>
__global__ void __launch_bounds__(256) ade_collide_kernel(const __grid_constant__ AdeK k,
                                                          const uint32_t* __restrict__ list, int64_t count) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane;
    const uint32_t N32 = (uint32_t)N;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < count; r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t n = list[r];
        const uint8_t dyn = k.cls[n] & 3;
        int x, y, z;
        decode(k.g, n, x, y, z);
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) { atomicAdd(&k.counters[1], 1ull); continue; }
        const float ux = k.u[n], uy = k.u[N + n], uz = k.u[2 * N + n];
        const bool adj = (x == 1 || x == k.g.nx - 2);
        for (int m = 0; m < p.n_mob; ++m) {
            float* pm = k.pop + (int64_t)m * 7 * N;
            float f[7];
            gather7<PARITY>(pm, N32, st, f);
            float rho = 0.f;
            if (dyn == BB) {
#pragma unroll
                for (int i = 1; i < 4; ++i) { const float tmp = f[i]; f[i] = f[i + 3]; f[i + 3] = tmp; }
            } else if (dyn != NODYN) {
                const float om = (dyn == BIO) ? p.omega_bio[m] : p.omega_pore[m];
                collide7(f, om, ux, uy, uz, rho);
            } else if (adj) {
#pragma unroll
                for (int i = 0; i < 7; ++i) rho += f[i];
            }
            if (adj && dyn != BB) {
                const int side = (x == 1) ? 0 : 1;
                k.rho_adj[((int64_t)m * 2 + side) * plane + (n - (int64_t)x * plane)] = rho;
            }
#pragma unroll
            for (int i = 0; i < 7; ++i) pm[slot7<PARITY>(N32, st, i)] = f[i];
        }
    }
}

// stream without collision: gather at this parity, scatter (the AA swap)
template <int PARITY>
__global__ void __launch_bounds__(256) ade_stream_only_kernel(const __grid_constant__ AdeK k,
                                                              const uint32_t* __restrict__ list, int64_t count) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N;
    const uint32_t N32 = (uint32_t)N;
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < count; r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t n = list[r];
        int x, y, z;
        decode(k.g, n, x, y, z);
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) { atomicAdd(&k.counters[1], 1ull); continue; }
        for (int m = 0; m < p.n_mob; ++m) {
            float* pm = k.pop + (int64_t)m * 7 * N;
            float f[7];
            gather7<PARITY>(pm, N32, st, f);
            scatter7<PARITY>(pm, N32, st, f);
        }
    }
}

template <int NMOB>
static int boundary_launch(Ctx* c, const AdeK& k) {
    const int bblocks = grid_for(2 * c->geo.plane, 256, 148 * 4);
    if (c->ade_parity == 0) ade_boundary_kernel<NMOB, 0><<<bblocks, 256, 0, c->stream>>>(k);
    else ade_boundary_kernel<NMOB, 1><<<bblocks, 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("ade_boundary_kernel");
    c->launches += 1;
    return CL_OK;
}

static int boundary(Ctx* c, const AdeK& k) {
    switch (c->ap.n_mob) {
        case 1: return boundary_launch<1>(c, k);
        case 2: return boundary_launch<2>(c, k);
        case 3: return boundary_launch<3>(c, k);
        case 4: return boundary_launch<4>(c, k);
        case 5: return boundary_launch<5>(c, k);
        case 6: return boundary_launch<6>(c, k);
        case 7: return boundary_launch<7>(c, k);
        case 8: return boundary_launch<8>(c, k);
        default: set_error("the per-operator entry points take 1..8 mobile solutes"); return CL_ERR_ARG;
    }
}

static int ops_prepare(Ctx* c) {
    int r = CL_OK;
    if (!c->ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
    if (c->ap.n_mob < 1 || c->ap.n_mob > 8) { set_error("the per-operator entry points take 1..8 mobile solutes"); return CL_ERR_ARG; }
    if (c->cfg.rate_law != CL_RATELAW_TABLE) {
        set_error("the per-operator entry points run the rate table; a compiled rate law runs in cl_step");
        return CL_ERR_STATE;
    }
    if (c->store_dirty && (r = store_update(c, 0))) return r;
    if (c->live_dirty && (r = build_live_list(c))) return r;
    return CL_OK;
}

// the step's counters: CL_WARN_NOT_CONVERGED when a Newton solve missed,
// an error when a site lacked storage
static int ops_finish(Ctx* c) {
    unsigned long long cnts[2] = {0, 0};
    CL_CUDA(cudaMemcpyAsync(cnts, c->d_counters, sizeof cnts, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaMemsetAsync(c->d_counters, 0, sizeof cnts, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    if (cnts[1]) { set_error("a live site's slots had no storage"); return CL_ERR_STATE; }
    return cnts[0] ? CL_WARN_NOT_CONVERGED : CL_OK;
}

int ops_collide(Ctx* c) {
    int r = ops_prepare(c);
    if (r) return r;
    if (c->op_collided) { set_error("cl_op_collide twice without cl_op_stream"); return CL_ERR_STATE; }
    AdeK k = make_adek(c);
    if (c->n_live > 0) {
        const int blocks = grid_for(c->n_live, 256, 148 * 8);
        if (c->ade_parity == 0) ade_collide_kernel<0><<<blocks, 256, 0, c->stream>>>(k, c->d_live, c->n_live);
        else ade_collide_kernel<1><<<blocks, 256, 0, c->stream>>>(k, c->d_live, c->n_live);
        CL_LAUNCH_CHECK("ade_collide_kernel");
        c->launches += 1;
    }
    c->op_collided = true;
    return ops_finish(c);
}

int ops_stream(Ctx* c) {
    int r = ops_prepare(c);
    if (r) return r;
    if (!c->op_collided) { set_error("cl_op_stream needs cl_op_collide first"); return CL_ERR_STATE; }
    AdeK k = make_adek(c);
    if (c->n_live > 0) {
        const int blocks = grid_for(c->n_live, 256, 148 * 8);
        if (c->ade_parity == 0) ade_stream_only_kernel<0><<<blocks, 256, 0, c->stream>>>(k, c->d_live, c->n_live);
        else ade_stream_only_kernel<1><<<blocks, 256, 0, c->stream>>>(k, c->d_live, c->n_live);
        CL_LAUNCH_CHECK("ade_stream_only_kernel");
        c->launches += 1;
    }
    if ((r = boundary(c, k))) return r;
    c->ade_parity ^= 1;
    c->op_collided = false;
    ++c->step_index;
    return ops_finish(c);
}

int ops_react(Ctx* c, int ops) {
    int r = ops_prepare(c);
    if (r) return r;
    AdeK k = make_adek(c);
    if ((ops & 4) && c->ap.do_dissol) {
        // the phase voxels' releases see the water after this step's
        // kinetics: recomputed from the current state when the kinetics run in
        // the same call, the current state itself otherwise
        AdeK kd = k;
        if (!(ops & 3)) { kd.p.do_kin = 0; kd.p.n_srg = 0; }
        if ((r = dissol_release(c, kd))) return r;
    }
    const int nc = c->ap.do_eq ? c->cfg.eq.n_comp : 0;
    switch (nc) {
        case 0: r = ade_ops_nc0(c, k, ops); break;
        case 1: r = ade_ops_nc1(c, k, ops); break;
        case 2: r = ade_ops_nc2(c, k, ops); break;
        case 3: r = ade_ops_nc3(c, k, ops); break;
        case 4: r = ade_ops_nc4(c, k, ops); break;
        case 5: r = ade_ops_nc5(c, k, ops); break;
        default: set_error("equilibrium in the transport step supports 1..5 components"); return CL_ERR_ARG;
    }
    if (r) return r;
    return ops_finish(c);
}

}  // namespace cl
