// geometry.cu -- node classes from the mask, the dynamics switch after a mask
// change, precipitation node conversion and the global reductions.  All
// integer/byte work: results are bit-exact against the oracle.
#include <vector>
#include "internal.h"

namespace cl {

struct ClassK {
    Geo g;
    const uint8_t* mask;
    uint8_t* ns;
    uint8_t* ade;
    int solid, bb;
    int n_pore, pore[CL_MAX_CODES];
    int n_bio, bio[CL_MAX_CODES];
    int bio_is_bb;                 // perm_ratio <= 1e-14: biofilm is BounceBack for the flow
    const uint8_t* phase;          // dissolvable phase ids (null without dissolution)
    unsigned long long* counts;    // [0] BGK flow sites, [1] coupled flow NoDyn, [2] coupled ade NoDyn
};

__device__ __forceinline__ bool in_codes(int v, const int* list, int n) {
    for (int i = 0; i < n; ++i) if (list[i] == v) return true;
    return false;
}

__device__ __forceinline__ bool is_wall(const ClassK& k, int m) { return m == k.solid || m == k.bb; }

// reactive: interior in x and not solid / bounce-back (processor guards of
// run_kinetics etc.); surface: a face neighbour is solid or bounce-back
// (surfaceAbioticKinetics3D, precipitationVOP.hh:79-90; y,z periodic here).
// Phase flags: the voxel carries a phase, or a face neighbour inside
// x = 1..nx-2 and inside y, z (no wrap: surfaceDissolutionKinetics3D,
// dissolutionVOP.hh:323-325) does.
__device__ uint8_t flags_for(const ClassK& k, int64_t n, int x, int y, int z) {
    const int m = k.mask[n];
    uint8_t fl = 0;
    if (x > 0 && x < k.g.nx - 1 && !is_wall(k, m)) fl |= F_REACTIVE;
    const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
    for (int d = 0; d < 6; ++d) {
        const int64_t q = nbr(k.g, n, x, y, z, d6[d][0], d6[d][1], d6[d][2]);
        if (q < 0) continue;
        if (is_wall(k, k.mask[q])) { fl |= F_SURFACE; break; }
    }
    if (k.phase) {
        if (k.phase[n]) fl |= F_PHASE_SELF;
        for (int d = 0; d < 6; ++d) {
            const int ax = x + d6[d][0], ay = y + d6[d][1], az = z + d6[d][2];
            if (ax < 1 || ax > k.g.nx - 2 || ay < 0 || ay >= k.g.ny || az < 0 || az >= k.g.nz) continue;
            if (k.phase[((int64_t)ax * k.g.ny + ay) * k.g.nz + az]) { fl |= F_PHASE_NBR; break; }
        }
    }
    return fl;
}

// NSdomainSetup / soluteDomainSetup dynamics assignment (complab_functions.hh:245-340)
__global__ void classes_kernel(ClassK k) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        const int m = k.mask[n];
        uint8_t ns = FLUID, ad = FLUID;
        if (in_codes(m, k.pore, k.n_pore)) { ns = FLUID; ad = FLUID; }
        if (k.bb > 0 && m == k.bb) { ns = BB; ad = BB; }
        if (k.solid >= 0 && m == k.solid) { ns = NODYN; ad = NODYN; }
        if (in_codes(m, k.bio, k.n_bio)) { ns = k.bio_is_bb ? BB : BIO; ad = BIO; }
        k.ns[n] = ns;
        k.ade[n] = ad | flags_for(k, n, x, y, z);
    }
}

// updateNsLatticesDynamics3D (part2.hh:630-695): a site whose flow dynamics is
// the pore IncBGK and whose mask is no longer a pore code becomes BounceBack
// (impermeable biofilm / precipitate) or IncBGK(omega_bio); a pore-coded site
// with any other dynamics returns to the pore IncBGK.
// updateSoluteDynamics3D (:461-529): non-wall sites switch their solute omega
// between pore and biofilm; wall-coded sites keep their solute dynamics.
__global__ void update_dynamics_kernel(ClassK k) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        const int m = k.mask[n];
        const bool pore = in_codes(m, k.pore, k.n_pore);
        uint8_t ns = k.ns[n];
        if (!pore && ns == FLUID) ns = k.bio_is_bb ? BB : BIO;
        else if (pore && ns != FLUID) ns = FLUID;
        k.ns[n] = ns;
        uint8_t ad = k.ade[n] & 3;
        if (!is_wall(k, m) && (ad == FLUID || ad == BIO)) ad = pore ? FLUID : BIO;
        k.ade[n] = ad | flags_for(k, n, x, y, z);
    }
}

// class flags only, after a mask or phase change that does not switch dynamics
// (the reaction processors read the mask every step)
__global__ void flags_kernel(ClassK k) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        k.ade[n] = (uint8_t)((k.ade[n] & 3) | flags_for(k, n, x, y, z));
    }
}

// Counts that steer the step kernels: BGK flow sites (energy average) and
// whether any NoDynamics site is linked to a dynamic site (otherwise NoDynamics
// regions are sealed behind bounce-back and need no streaming at all).  A
// NoDynamics or bounce-back solute site whose mask reopened to pore reacts,
// and what it adds reaches NoDynamics neighbours too, so it counts as a link.
__global__ void class_counts_kernel(ClassK k) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long nb = 0, cf = 0, ca = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        const uint8_t ns = k.ns[n], ad = k.ade[n] & 3;
        if (ns == FLUID || ns == BIO) ++nb;
        // a wall-class solute site whose mask reopened reacts, and its
        // increments stream into NoDynamics neighbours as well
        const bool reopened = (ad == NODYN || ad == BB) && (k.ade[n] & F_REACTIVE);
        if (reopened) ++ca;
        if (ns != NODYN && ad != NODYN) continue;
        int x, y, z;
        decode(k.g, n, x, y, z);
        if (ns == NODYN) {
            for (int i = 1; i < 19; ++i) {
                const int64_t q = nbr(k.g, n, x, y, z, c19x(i), c19y(i), c19z(i));
                if (q < 0) continue;
                const uint8_t c = k.ns[q];
                if (c == FLUID || c == BIO) { ++cf; break; }
            }
        }
        if (ad == NODYN && !reopened) {
            for (int i = 1; i < 7; ++i) {
                const int64_t q = nbr(k.g, n, x, y, z, c7x(i), c7y(i), c7z(i));
                if (q < 0) continue;
                const uint8_t c = k.ade[q] & 3;
                if (c == FLUID || c == BIO) { ++ca; break; }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        nb += __shfl_down_sync(0xffffffffu, nb, o);
        cf += __shfl_down_sync(0xffffffffu, cf, o);
        ca += __shfl_down_sync(0xffffffffu, ca, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (nb) atomicAdd(&k.counts[0], nb);
        if (cf) atomicAdd(&k.counts[1], cf);
        if (ca) atomicAdd(&k.counts[2], ca);
    }
}

static ClassK make_classk(Ctx* c) {
    ClassK k;
    k.g = c->geo;
    k.mask = c->d_mask;
    k.ns = c->d_ns_cls;
    k.ade = c->d_ade_cls;
    k.solid = c->cfg.solid_code;
    k.bb = c->cfg.bb_code;
    k.n_pore = c->cfg.n_pore_codes;
    k.n_bio = c->cfg.n_bio_codes;
    for (int i = 0; i < CL_MAX_CODES; ++i) { k.pore[i] = c->cfg.pore_codes[i]; k.bio[i] = c->cfg.bio_codes[i]; }
    k.bio_is_bb = c->cfg.perm_ratio > 1e-14 ? 0 : 1;
    k.phase = c->d_phase;
    k.counts = reinterpret_cast<unsigned long long*>(c->d_scratch);
    return k;
}

static int refresh_counts(Ctx* c, ClassK& k) {
    CL_CUDA(cudaMemsetAsync(k.counts, 0, 3 * sizeof(unsigned long long), c->stream));
    class_counts_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("class_counts_kernel");
    unsigned long long h[3];
    CL_CUDA(cudaMemcpyAsync(h, k.counts, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    c->n_bgk = (int64_t)h[0];
    c->flow_nodyn_coupled = h[1] > 0;
    c->ade_nodyn_coupled = h[2] > 0;
    c->live_dirty = true;
    c->flive_dirty = true;
    c->store_dirty = true;
    c->fstore_dirty = true;
    return CL_OK;
}

// The live list: interior sites whose transport class streams (not a
// bounce-back site, unless its mask reopened; a NoDynamics site only when
// NoDynamics sites stream), in increasing site order: the streaming launch
// runs one thread per entry, the reaction launch the reactive entries.  Each of kListBlocks blocks owns one contiguous chunk of sites:
// pass 1 counts, the host scans the counts, pass 2 writes in order.
constexpr int kListBlocks = 148 * 8;

__device__ __forceinline__ bool live_site(uint8_t cls, int nodyn_coupled) {
    const uint8_t dyn = cls & 3;
    return !((dyn == BB && !(cls & F_REACTIVE)) || (dyn == NODYN && !nodyn_coupled));
}

__global__ void live_count_kernel(const uint8_t* cls, int64_t lo, int64_t hi, int64_t chunk, int nodyn_coupled,
                                   int64_t* counts) {
    __shared__ int64_t s_part[8];
    const int64_t b0 = lo + (int64_t)blockIdx.x * chunk, b1 = min(hi, b0 + chunk);
    int64_t cnt = 0;
    for (int64_t n = b0 + threadIdx.x; n < b1; n += blockDim.x) cnt += live_site(cls[n], nodyn_coupled);
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_part[w];
        counts[blockIdx.x] = t;
    }
}

// blockDim.x == 256: the chunk is walked in rounds of 256 sites, each round's
// hits placed by a block-wide ballot scan
__global__ void live_write_kernel(const uint8_t* cls, int64_t lo, int64_t hi, int64_t chunk, int nodyn_coupled,
                                   const int64_t* offsets, uint32_t* list) {
    __shared__ int s_warp[8];
    __shared__ int64_t s_base;
    const int64_t b0 = lo + (int64_t)blockIdx.x * chunk, b1 = min(hi, b0 + chunk);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (threadIdx.x == 0) s_base = offsets[blockIdx.x];
    __syncthreads();
    for (int64_t r0 = b0; r0 < b1; r0 += blockDim.x) {
        const int64_t n = r0 + threadIdx.x;
        const bool hit = n < b1 && live_site(cls[n], nodyn_coupled);
        const unsigned ball = __ballot_sync(0xffffffffu, hit);
        if (lane == 0) s_warp[w] = __popc(ball);
        __syncthreads();
        int before = 0, total = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { if (q < w) before += s_warp[q]; total += s_warp[q]; }
        if (hit) list[s_base + before + __popc(ball & ((1u << lane) - 1u))] = (uint32_t)n;
        __syncthreads();
        if (threadIdx.x == 0) s_base += total;
        __syncthreads();
    }
}

// lower_bound of each site bound in the sorted live list (in place)
__global__ void live_bounds_kernel(const uint32_t* list, int64_t count, int64_t* bounds, int nb) {
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const int64_t key = bounds[j];
        int64_t a = 0, b = count;
        while (a < b) {
            const int64_t mid = (a + b) >> 1;
            if ((int64_t)list[mid] < key) a = mid + 1; else b = mid;
        }
        bounds[j] = a;
    }
}

// the sites of [lo, hi) whose class byte passes live_site, in site order,
// into *list (allocated once with capacity hi - lo); *count their number
static int compact_sites(Ctx* c, const uint8_t* cls, int64_t lo, int64_t hi, int coupled, uint32_t** list,
                         int64_t* count) {
    const int64_t chunk = (hi - lo + kListBlocks - 1) / kListBlocks;
    if (!c->d_live_blk) { int r = dalloc(c, &c->d_live_blk, (size_t)kListBlocks); if (r) return r; }
    live_count_kernel<<<kListBlocks, 256, 0, c->stream>>>(cls, lo, hi, chunk, coupled, c->d_live_blk);
    CL_LAUNCH_CHECK("live_count_kernel");
    std::vector<int64_t> h(kListBlocks);
    CL_CUDA(cudaMemcpyAsync(h.data(), c->d_live_blk, sizeof(int64_t) * kListBlocks, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    int64_t total = 0;
    for (int b = 0; b < kListBlocks; ++b) { const int64_t v = h[b]; h[b] = total; total += v; }
    if (!*list) {
        // capacity for every site of the range: the list never needs a reallocation
        int r = dalloc(c, list, (size_t)(hi - lo));
        if (r) return r;
    }
    CL_CUDA(cudaMemcpyAsync(c->d_live_blk, h.data(), sizeof(int64_t) * kListBlocks, cudaMemcpyHostToDevice, c->stream));
    live_write_kernel<<<kListBlocks, 256, 0, c->stream>>>(cls, lo, hi, chunk, coupled, c->d_live_blk, *list);
    CL_LAUNCH_CHECK("live_write_kernel");
    CL_CUDA(cudaStreamSynchronize(c->stream));   // h is read by the copy above
    *count = total;
    return CL_OK;
}

// The flow's list: every site that is not bounce-back (a no-op of the AA
// step) and not an uncoupled NoDynamics site, boundary planes included.  The
// flow class byte carries no flags, so live_site reads it as it is.
int build_flow_list(Ctx* c) {
    int r = compact_sites(c, c->d_ns_cls, 0, c->geo.N, c->flow_nodyn_coupled ? 1 : 0, &c->d_flive, &c->n_flive);
    if (r) return r;
    c->flive_dirty = false;
    return CL_OK;
}

int build_live_list(Ctx* c) {
    const int64_t lo = c->geo.plane, hi = c->geo.N - c->geo.plane;   // interior x
    int r = compact_sites(c, c->d_ade_cls, lo, hi, c->ade_nodyn_coupled ? 1 : 0, &c->d_live, &c->n_live);
    if (r) return r;
    const int64_t total = c->n_live;
    // slab boundaries: whole x planes; each slab's first list entry by binary search
    const int G = c->slabs;
    const int64_t planes = c->geo.nx - 2;
    for (int j = 0; j <= G; ++j) c->slab_site[j] = lo + (planes * j / G) * c->geo.plane;
    int64_t* d_b = c->d_live_blk;                    // reuse: G+1 bounds in, offsets out
    CL_CUDA(cudaMemcpyAsync(d_b, c->slab_site, sizeof(int64_t) * (G + 1), cudaMemcpyHostToDevice, c->stream));
    live_bounds_kernel<<<1, 128, 0, c->stream>>>(c->d_live, total, d_b, G + 1);
    CL_LAUNCH_CHECK("live_bounds_kernel");
    CL_CUDA(cudaMemcpyAsync(c->slab_live, d_b, sizeof(int64_t) * (G + 1), cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    c->live_dirty = false;
    return CL_OK;
}

int classes_from_mask(Ctx* c) {
    ClassK k = make_classk(c);
    classes_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("classes_kernel");
    return refresh_counts(c, k);
}

int refresh_flags(Ctx* c) {
    ClassK k = make_classk(c);
    flags_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("flags_kernel");
    return refresh_counts(c, k);
}

int update_dynamics(Ctx* c) {
    ClassK k = make_classk(c);
    update_dynamics_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("update_dynamics_kernel");
    return refresh_counts(c, k);
}

// precipNodeConversion3D (precipitationVOP.hh:158-219): a non-wall site whose
// precipitate inventory reached max_precipRho takes the precipitate code, and
// the precipitate phase id when one is declared (so it can dissolve later).
__global__ void precip_kernel(Geo g, uint8_t* mask, const double* inv, double thr, int solid, int bb,
                              int code, uint8_t* phase, int phase_id, unsigned long long* changed) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long cnt = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        const int m = mask[n];
        if (m == solid || m == bb) continue;
        if (inv[n] >= thr) {
            if (m != code) ++cnt;
            mask[n] = (uint8_t)code;
            if (phase && phase_id > 0) phase[n] = (uint8_t)phase_id;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(changed, cnt);
}

int precip_convert(Ctx* c, int64_t* changed) {
    const int s = c->cfg.precip_substrate;
    if (s < 0 || s >= c->ap.S || c->ap.mob_slot[s] >= 0) {
        set_error("precipitation needs an immobile precipitate substrate");
        return CL_ERR_ARG;
    }
    unsigned long long* d_cnt = reinterpret_cast<unsigned long long*>(c->d_scratch);
    CL_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), c->stream));
    precip_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(
        c->geo, c->d_mask, c->d_imm + (int64_t)s * c->geo.N, c->cfg.max_precip_rho,
        c->cfg.solid_code, c->cfg.bb_code, c->cfg.precip_code, c->d_phase, c->cfg.precip_phase_id, d_cnt);
    CL_LAUNCH_CHECK("precip_kernel");
    unsigned long long h = 0;
    CL_CUDA(cudaMemcpyAsync(&h, d_cnt, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    *changed = (int64_t)h;
    return h ? refresh_flags(c) : CL_OK;
}

// initPhaseLattice3D (dissolutionVOP.hh:195-229): a site takes the id of the
// first grain (not precipitate) phase whose material is its mask code.
struct PhaseTab {
    int n;
    int material[CL_MAX_PHASES], substrate[CL_MAX_PHASES], is_precip[CL_MAX_PHASES];
    double full[CL_MAX_PHASES], fill[CL_MAX_PHASES];
};

static PhaseTab make_phasetab(const Ctx* c) {
    PhaseTab t{};
    t.n = c->cfg.n_phases;
    for (int k = 0; k < t.n; ++k) {
        const cl_phase& ph = c->cfg.phases[k];
        t.material[k] = ph.material; t.substrate[k] = ph.substrate; t.is_precip[k] = ph.is_precipitate;
        t.full[k] = ph.full_density; t.fill[k] = ph.initial_fill;
    }
    return t;
}

__global__ void phase_seed_kernel(Geo g, const uint8_t* mask, uint8_t* phase, PhaseTab t) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        const int m = mask[n];
        uint8_t pid = 0;
        for (int k = 0; k < t.n; ++k)
            if (!t.is_precip[k] && t.material[k] == m) { pid = (uint8_t)(k + 1); break; }
        phase[n] = pid;
    }
}

int phase_seed(Ctx* c) {
    if (!c->d_phase) return CL_OK;
    phase_seed_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(c->geo, c->d_mask, c->d_phase, make_phasetab(c));
    CL_LAUNCH_CHECK("phase_seed_kernel");
    return CL_OK;
}

// each grain phase with initial_fill > 0 seeds that inventory on its material
// (initializeScalarLattice3D, complab.cpp:858-871), phases in declaration order
__global__ void phase_fill_kernel(Geo g, const uint8_t* mask, double* imm, PhaseTab t) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        const int m = mask[n];
        for (int k = 0; k < t.n; ++k)
            if (!t.is_precip[k] && t.fill[k] > 0.0 && t.material[k] == m) imm[(int64_t)t.substrate[k] * g.N + n] = t.fill[k];
    }
}

int phase_fill(Ctx* c) {
    if (!c->d_phase) return CL_OK;
    phase_fill_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(c->geo, c->d_mask, c->d_imm, make_phasetab(c));
    CL_LAUNCH_CHECK("phase_fill_kernel");
    return CL_OK;
}

// dissolNodeConversion3D (dissolutionVOP.hh:459-527): a phase site whose
// mineral fell below reopen_fraction * full_density takes the pore code and
// loses its phase id.
__global__ void dissol_convert_kernel(Geo g, uint8_t* mask, uint8_t* phase, const double* imm, PhaseTab t,
                                      double reopen, int pore, unsigned long long* changed) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long cnt = 0;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        const int pid = phase[n];
        if (pid <= 0 || pid > t.n) continue;
        const int k = pid - 1;
        if (!(t.full[k] > 0.0)) continue;
        const double mineral = imm[(int64_t)t.substrate[k] * g.N + n];
        if (mineral < reopen * t.full[k]) {
            if (mask[n] != pore) ++cnt;
            mask[n] = (uint8_t)pore;
            phase[n] = 0;
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(changed, cnt);
}

int dissol_convert(Ctx* c, int64_t* changed) {
    *changed = 0;
    if (!c->d_phase) { set_error("dissolution is not enabled in this context"); return CL_ERR_STATE; }
    const int pore = c->cfg.n_pore_codes > 0 ? c->cfg.pore_codes[0] : 2;
    unsigned long long* d_cnt = reinterpret_cast<unsigned long long*>(c->d_scratch);
    CL_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), c->stream));
    dissol_convert_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(
        c->geo, c->d_mask, c->d_phase, c->d_imm, make_phasetab(c), c->cfg.reopen_fraction, pore, d_cnt);
    CL_LAUNCH_CHECK("dissol_convert_kernel");
    unsigned long long h = 0;
    CL_CUDA(cudaMemcpyAsync(&h, d_cnt, sizeof h, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    *changed = (int64_t)h;
    return h ? refresh_flags(c) : CL_OK;
}

// Deterministic FP64 reduction: fixed-size grid, per-block partials, one final
// block summing them in index order.
__global__ void reduce_part_kernel(const double* v, int64_t n, int op, double* part) {
    __shared__ double red[256];
    double acc = (op == CL_RED_SUM) ? 0.0 : (op == CL_RED_MIN ? 1.0 / 0.0 : -1.0 / 0.0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = v[i];
        acc = (op == CL_RED_SUM) ? acc + x : (op == CL_RED_MIN ? fmin(acc, x) : fmax(acc, x));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double a = red[threadIdx.x], b = red[threadIdx.x + o];
            red[threadIdx.x] = (op == CL_RED_SUM) ? a + b : (op == CL_RED_MIN ? fmin(a, b) : fmax(a, b));
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void count_eq_kernel(const uint8_t* mask, int64_t n, int code, unsigned long long* out) {
    unsigned long long cnt = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        cnt += (mask[i] == code);
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(out, cnt);
}

int reduce_field(Ctx* c, const double* d_field, int op, double arg, const uint8_t* d_mask, double* out) {
    if (op == CL_RED_COUNT_EQ) {
        unsigned long long* d_cnt = reinterpret_cast<unsigned long long*>(c->d_scratch);
        CL_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long), c->stream));
        count_eq_kernel<<<grid_for(c->geo.N, 256, 148 * 8), 256, 0, c->stream>>>(d_mask, c->geo.N, (int)arg, d_cnt);
        CL_LAUNCH_CHECK("count_eq_kernel");
        unsigned long long h = 0;
        CL_CUDA(cudaMemcpyAsync(&h, d_cnt, sizeof h, cudaMemcpyDeviceToHost, c->stream));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        *out = (double)h;
        return CL_OK;
    }
    const int blocks = 148 * 4;
    double* part = c->d_scratch;
    reduce_part_kernel<<<blocks, 256, 0, c->stream>>>(d_field, c->geo.N, op, part);
    reduce_part_kernel<<<1, 256, 0, c->stream>>>(part, blocks, op, part + blocks);
    CL_LAUNCH_CHECK("reduce_part_kernel");
    CL_CUDA(cudaMemcpyAsync(out, part + blocks, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

}  // namespace cl
