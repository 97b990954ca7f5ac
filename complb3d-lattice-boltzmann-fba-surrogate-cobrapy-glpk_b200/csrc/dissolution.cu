// dissolution.cu -- mineral release of the dissolvable phases
// (surfaceDissolutionKinetics3D, src/dissolutionVOP.hh:265-435).
//
// One thread per phase voxel in x = 1..nx-2.  Its open faces are the face
// neighbours inside x = 1..nx-2 and inside y, z (no wrap) whose mask is not
// solid or bounce-back; the water it sees is the mean solute density over them
// after this step's kinetics, which the reference applies before dissolution
// runs (complab.cpp:1252-1318), so the thread recomputes the kinetics
// increments of each open neighbour from the same pre-step state the fused
// kernel starts from.  The rate law is the table of cl_phase; at most half the
// mineral goes per step and the products scale with it.  The result is stored
// per phase voxel in rel[S][N]: the products per open face (zero where
// |released| <= thrd) and, at the phase substrate, the voxel's own decrement.
// The fused kernel gathers those records; a decrement on a solid or
// bounce-back voxel is dropped as update_abiotic_rxnLattices drops it, or with
// dissol_apply_at_walls applied here (the voxel's inventory is read by no
// other thread of this launch).
#include "ade_kernels.cuh"

namespace cl {

template <int NMOB, int PARITY>
__device__ __forceinline__ void voxel_densities(const AdeK& k, int x, int y, int z, uint32_t n, double* C) {
    const AdeParams& p = k.p;
    SSite st;
    if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) atomicAdd(&k.counters[1], 1ull);
    const uint32_t N32 = (uint32_t)k.g.N;
#pragma unroll
    for (int m = 0; m < NMOB; ++m) {
        float f[7];
        gather7<PARITY>(k.pop + (int64_t)m * 7 * k.g.N, N32, st, f);
        float r = 0.f;
#pragma unroll
        for (int i = 0; i < 7; ++i) r += f[i];
        C[p.mob_index[m]] = (double)r;
    }
    for (int s = 0; s < p.S; ++s)
        if (p.mob_slot[s] < 0) C[s] = k.imm[(int64_t)s * k.g.N + n];
}

// densities after the kinetics increments of this step (update_rxnLattices)
template <int NMOB, int PARITY>
__device__ __forceinline__ void post_kinetics(const AdeK& k, int x, int y, int z, uint32_t n, double* C) {
    const AdeParams& p = k.p;
    voxel_densities<NMOB, PARITY>(k, x, y, z, n, C);
    if (p.do_kin || p.n_srg > 0) {
        double R[CL_MAX_SOLUTES], B[CL_MAX_MICROBES], BR[CL_MAX_MICROBES];
        kinetics_increments(p, k.bio, k.g.N, n, C, 1, R, B, BR, 1);
        for (int s = 0; s < p.S; ++s) {
            const double d = R[s];
            if (d > THRD || d < -THRD) C[s] += d;
        }
    }
}

template <int NMOB, int PARITY>
__global__ void __launch_bounds__(128) dissol_release_kernel(const __grid_constant__ AdeK k) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane;
    const int nx = k.g.nx, ny = k.g.ny, nz = k.g.nz;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = plane + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < N - plane; n += stride) {
        const int pid = k.phase[n];
        if (pid == 0) continue;
        const cl_phase& ph = p.phase[pid - 1];
        const int sM = ph.substrate;
        for (int s = 0; s < p.S; ++s) k.rel[(int64_t)s * N + n] = 0.0;
        int x, y, z;
        decode(k.g, n, x, y, z);
        const bool reactive = (k.cls[n] & F_REACTIVE) != 0;
        double C[CL_MAX_SOLUTES];
        double mineral;
        if (reactive && (p.do_kin || p.n_srg > 0)) {
            post_kinetics<NMOB, PARITY>(k, x, y, z, (uint32_t)n, C);
            mineral = C[sM];
        } else {
            mineral = k.imm[(int64_t)sM * N + n];
        }
        if (!(mineral > THRD)) continue;
        // open faces, in the reference's direction order +x -x +y -y +z -z
        const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
        int n_open = 0;
        double water[CL_MAX_SOLUTES];
        for (int s = 0; s < p.S; ++s) water[s] = 0.0;
        for (int d = 0; d < 6; ++d) {
            const int ax = x + d6[d][0], ay = y + d6[d][1], az = z + d6[d][2];
            if (ax < 1 || ax > nx - 2 || ay < 0 || ay >= ny || az < 0 || az >= nz) continue;
            const uint32_t q = (uint32_t)(((int64_t)ax * ny + ay) * nz + az);
            const int m = k.mask[q];
            if (m == p.solid_code || m == p.bb_code) continue;
            ++n_open;
            post_kinetics<NMOB, PARITY>(k, ax, ay, az, q, C);
            for (int s = 0; s < p.S; ++s) water[s] += C[s];
        }
        if (n_open == 0 && p.dissol_surface_only) continue;
        if (n_open > 0)
            for (int s = 0; s < p.S; ++s) water[s] /= (double)n_open;
        for (int s = 0; s < p.S; ++s) if (water[s] < 0.0) water[s] = 0.0;
        // the rate law of the phase (defineDissolutionRate as a table)
        double rate = ph.k * fmax(mineral, 0.0);
        for (int j = 0; j < ph.n_mass; ++j) rate *= water[ph.mass_s[j]];
        const double mineral_r = isfinite(rate) ? -rate : 0.0;
        if (!(mineral_r < 0.0)) continue;
        double dm = mineral_r * p.dt;
        double scale = 1.0;
        const double max_remove = 0.5 * mineral;
        if (-dm > max_remove) scale = max_remove / (-dm);
        dm *= scale;
        if (!(-dm > THRD)) continue;
        if (reactive) k.rel[(int64_t)sM * N + n] = dm;
        else if (p.dissol_walls) k.imm[(int64_t)sM * N + n] += dm;
        if (n_open == 0) continue;
        for (int s = 0; s < p.S; ++s) {
            if (s == sM) continue;
            double sr = ph.nu[s] * rate;
            if (!isfinite(sr)) sr = 0.0;
            const double released = sr * p.dt * scale;
            if (fabs(released) <= THRD) continue;
            k.rel[(int64_t)s * N + n] = released / (double)n_open;
        }
    }
}

template <int NMOB>
static int launch_release(Ctx* c, const AdeK& k) {
    const int64_t interior = c->geo.N - 2 * c->geo.plane;
    const int blocks = grid_for(interior, 128, 148 * 8);
    if (c->ade_parity == 0) dissol_release_kernel<NMOB, 0><<<blocks, 128, 0, c->stream>>>(k);
    else dissol_release_kernel<NMOB, 1><<<blocks, 128, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("dissol_release_kernel");
    c->launches += 1;
    return CL_OK;
}

int dissol_release(Ctx* c, const AdeK& k) {
    switch (c->ap.n_mob) {
        case 1: return launch_release<1>(c, k);
        case 2: return launch_release<2>(c, k);
        case 3: return launch_release<3>(c, k);
        case 4: return launch_release<4>(c, k);
        case 5: return launch_release<5>(c, k);
        case 6: return launch_release<6>(c, k);
        case 7: return launch_release<7>(c, k);
        case 8: return launch_release<8>(c, k);
        default: set_error("the fused transport step supports 1..8 mobile solutes");
                 return CL_ERR_ARG;
    }
}

}  // namespace cl
