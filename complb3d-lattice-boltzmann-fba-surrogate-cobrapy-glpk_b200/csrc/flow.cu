// flow.cu -- D3Q19 incompressible BGK flow on the AA pattern.
//
// Replaces Palabos IncBGKdynamics + collideAndStream as the reference drives it
// (NSdomainSetup, src/complab_functions.hh:245-294; loops src/complab.cpp:596-695).
// Populations are FP32 deviations fbar_i = f_i - t_i (the rho-1 storage the
// reference's processors assume), one 4-byte slot per population per site:
// 76 B read + 76 B write per fluid site per step.  The pressure boundaries on
// the x faces (regularized density boundary) and the energy reduction that
// drives the convergence tracer are fused into the same kernel.
//
// Slots are stored compactly: the sites that stream and their 18 D3Q19
// neighbours get storage indices in site order (fsidx; population arrays keep
// the stride N), so the slots of a run of pore sites are contiguous and a
// warp's loads fill whole sectors instead of fetching the solid sites' slots at
// the ends of every run.  An unstored site's slots read as 0, the value the
// full-lattice layout holds there (flow_init gives non-BGK sites 0 and nothing
// writes a slot no streaming site reaches).
#include "internal.h"
#include <cmath>

namespace cl {

struct FlowK {
    Geo g;
    float* f;
    const uint8_t* cls;
    float omega, omega_bio;
    float rb_in, rb_out;        // rhoBar at x = 0 and x = nx-1
    int nodyn_coupled;
    double* part;               // per-block energy partial sums
    const FlowTracer* tracer;   // early exit once converged (may be null)
    const uint32_t* list;       // the sites that stream, increasing
    int64_t count;
    const int32_t* sidx;        // N storage index of each site's slots (-1: none, reads 0)
    unsigned long long* counters;   // [2] streaming sites without the storage they need
};

// Palabos bgk_ma2_equilibrium with invRho = 1, deviation form
__device__ __forceinline__ float feq19(int i, float rb, float jx, float jy, float jz, float jsq) {
    float cj = c19x(i) * jx + c19y(i) * jy + c19z(i) * jz;
    return t19(i) * (rb + 3.f * cj + 4.5f * cj * cj - 1.5f * jsq);
}

// Regularized density boundary on an x face (side -1: x = 0, +1: x = nx-1).
// Normal momentum from the known populations, tangential momentum zero,
// PiNeq from the known populations counting the bounce-back of the unknown
// non-equilibrium parts, populations rebuilt as feq + t_i*9/2*Q_i:PiNeq.
template <int SIDE>
__device__ __forceinline__ void regularize(float* f, float rb, float& jx) {
    float s0 = 0.f, sn = 0.f;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        if (c19x(i) == 0) s0 += f[i];
        else if (c19x(i) == SIDE) sn += f[i];
    }
    jx = (SIDE < 0) ? (rb - s0 - 2.f * sn) : (s0 + 2.f * sn - rb);
    const float jsq = jx * jx;
    float pxx = 0, pyy = 0, pzz = 0, pxy = 0, pxz = 0, pyz = 0;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        if (c19x(i) == -SIDE) continue;
        const float w = (c19x(i) == 0) ? 1.f : 2.f;
        const float fn = w * (f[i] - feq19(i, rb, jx, 0.f, 0.f, jsq));
        const float cx = c19x(i), cy = c19y(i), cz = c19z(i);
        pxx += cx * cx * fn; pyy += cy * cy * fn; pzz += cz * cz * fn;
        pxy += cx * cy * fn; pxz += cx * cz * fn; pyz += cy * cz * fn;
    }
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        const float cx = c19x(i), cy = c19y(i), cz = c19z(i);
        const float cs2 = 1.f / 3.f;
        const float q = (cx * cx - cs2) * pxx + (cy * cy - cs2) * pyy + (cz * cz - cs2) * pzz
                      + 2.f * (cx * cy * pxy + cx * cz * pxz + cy * cz * pyz);
        f[i] = feq19(i, rb, jx, 0.f, 0.f, jsq) + t19(i) * 4.5f * q;
    }
}

// Storage indices of a site's slots: sl[0] its own, sl[i] that of the site at
// +c_i (its own where x leaves the lattice; that slot is reflected, never
// read there).  Returns false, with in-bounds substitutes, if one is missing.
template <int PARITY>
__device__ __forceinline__ bool flow_slots(const FlowK& k, const Site& st, uint32_t* sl) {
    bool ok = true;
    const int32_t s0 = k.sidx[st.n];
    if (s0 < 0) ok = false;
    sl[0] = s0 < 0 ? 0u : (uint32_t)s0;
    if (PARITY == 1) {
#pragma unroll
        for (int i = 1; i < 19; ++i) {
            uint32_t v = sl[0];
            if (st.inx(c19x(i))) {
                const int32_t q = k.sidx[st.at(c19x(i), c19y(i), c19z(i))];
                if (q < 0) ok = false;
                else v = (uint32_t)q;
            }
            sl[i] = v;
        }
    }
    return ok;
}

// AA pattern on the storage: even parity reads slot i of the site and writes
// slot opp(i); odd parity reads slot opp(i) of the upstream neighbour and
// writes slot i of the downstream one (x faces reflect into the own slots).
template <int PARITY>
__device__ __forceinline__ void gather19(const FlowK& k, const Site& st, const uint32_t* sl, float* f) {
    const uint32_t N = (uint32_t)k.g.N;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        if (PARITY == 0 || !st.inx(-c19x(i))) f[i] = k.f[i * N + sl[0]];
        else f[i] = k.f[opp19(i) * N + sl[opp19(i)]];
    }
}

template <int PARITY>
__device__ __forceinline__ void scatter19(const FlowK& k, const Site& st, const uint32_t* sl, const float* f) {
    const uint32_t N = (uint32_t)k.g.N;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        if (PARITY == 0 || !st.inx(c19x(i))) k.f[opp19(i) * N + sl[0]] = f[i];
        else k.f[i * N + sl[i]] = f[i];
    }
}

// the same gather for any site, stored or not (field output, statistics)
template <int PARITY>
__device__ __forceinline__ void gather19_any(const FlowK& k, const Site& st, float* f) {
    const uint32_t N = (uint32_t)k.g.N;
#pragma unroll
    for (int i = 0; i < 19; ++i) {
        const bool own = PARITY == 0 || !st.inx(-c19x(i));
        const int32_t s = k.sidx[own ? st.n : st.at(-c19x(i), -c19y(i), -c19z(i))];
        f[i] = s < 0 ? 0.f : k.f[(own ? i : opp19(i)) * N + (uint32_t)s];
    }
}

__device__ __forceinline__ Site site_of(const Geo& g, int64_t n) {
    int x, y, z;
    decode(g, n, x, y, z);
    return make_site(g, x, y, z, (uint32_t)n);
}

// One site of the collide-stream; returns 0.5|j|^2 for BGK sites.
template <int PARITY>
__device__ __forceinline__ double flow_site(const FlowK& k, const Site& st, int x, uint8_t cls) {
    float f[19];
    uint32_t sl[19];
    if (!flow_slots<PARITY>(k, st, sl)) atomicAdd(&k.counters[2], 1ull);
    gather19<PARITY>(k, st, sl, f);
    double e = 0.0;
    if (cls != NODYN) {
        const float om = (cls == BIO) ? k.omega_bio : k.omega;
        float rb, jx, jy = 0.f, jz = 0.f;
        if (x == 0) { rb = k.rb_in; regularize<-1>(f, rb, jx); }
        else if (x == k.g.nx - 1) { rb = k.rb_out; regularize<1>(f, rb, jx); }
        else {
            rb = 0.f; jx = 0.f;
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                rb += f[i];
                jx += c19x(i) * f[i]; jy += c19y(i) * f[i]; jz += c19z(i) * f[i];
            }
        }
        const float jsq = jx * jx + jy * jy + jz * jz;
#pragma unroll
        for (int i = 0; i < 19; ++i) f[i] = f[i] * (1.f - om) + om * feq19(i, rb, jx, jy, jz, jsq);
        e = 0.5 * (double)jsq;
    }
    scatter19<PARITY>(k, st, sl, f);
    return e;
}

// One thread per entry of the flow's site list (bounce-back sites, a no-op
// of the AA step, and uncoupled NoDynamics sites are not on it), so every
// lane of a warp has loads in flight.
template <int PARITY>
__global__ void __launch_bounds__(256, 3) flow_aa_kernel(FlowK k) {
    if (k.tracer && k.tracer->converged) return;
    double esum = 0.0;
    // the next list entry is loaded one iteration ahead, so a site's storage
    // lookups wait on one round trip to memory less (0.553 -> 0.529 ms at
    // 512x256x256)
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t n_next = r0 < k.count ? k.list[r0] : 0u;
    for (int64_t r = r0; r < k.count; r += stride) {
        const uint32_t n = n_next;
        if (r + stride < k.count) n_next = k.list[r + stride];
        int x, y, z;
        decode(k.g, n, x, y, z);
        esum += flow_site<PARITY>(k, make_site(k.g, x, y, z, n), x, k.cls[n]);
    }
    // deterministic block reduction of the energy
    __shared__ double red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) esum += __shfl_down_sync(0xffffffffu, esum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = esum;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        k.part[blockIdx.x] = s;
    }
}

// Sum the per-block partials in a fixed order and advance the ValueTracer.
__global__ void flow_finalize_kernel(const double* part, int nblocks, double inv_count,
                                     FlowTracer* tr, int use_tracer) {
    __shared__ double red[512];
    if (tr->converged) return;
    double s = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += part[b];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const double e = red[0] * inv_count;
    tr->last_energy = e;
    tr->steps_done += 1;
    if (!use_tracer) return;
    tr->window[tr->head] = e;
    tr->head = (tr->head + 1) % 500;
    if (tr->count < 500) tr->count += 1;
    if (tr->count >= 500) {
        double avg = 0.0;
        for (int i = 0; i < 500; ++i) avg += tr->window[i];
        avg /= 500.0;
        double sq = 0.0;
        for (int i = 0; i < 500; ++i) { double d = tr->window[i] - avg; sq += d * d; }
        const double ratio = sqrt(sq / 499.0) / avg;
        if (isnan(ratio)) { tr->diverged = 1; tr->converged = 1; tr->converged_at = tr->steps_done; }
        else if (ratio < tr->eps) { tr->converged = 1; tr->converged_at = tr->steps_done; }
    }
}

static FlowK make_flowk(Ctx* c) {
    FlowK k;
    k.g = c->geo;
    k.f = c->d_f;
    k.cls = c->d_ns_cls;
    const double om = 1.0 / c->cfg.tau_ns;
    k.omega = (float)om;
    k.omega_bio = (float)(1.0 / (c->cfg.perm_ratio * (1.0 / om - 0.5) + 0.5));
    k.rb_in = (float)(c->cfg.rho_in - 1.0);
    k.rb_out = (float)(c->cfg.rho_out - 1.0);
    k.nodyn_coupled = c->flow_nodyn_coupled ? 1 : 0;
    k.part = c->d_energy_part;
    k.tracer = c->d_tracer;
    k.list = nullptr;
    k.count = 0;
    k.sidx = c->d_fsidx;
    k.counters = c->d_counters;
    return k;
}

// initializeAtEquilibrium with the linear density profile into the stored
// slots; non-BGK sites hold 0 (BGK sites stream, so they are all stored).
__global__ void flow_init_kernel(Geo g, float* f, const int32_t* sidx, const uint8_t* cls, double rho_in,
                                 double rho_out) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        const int32_t s = sidx[n];
        if (s < 0) continue;
        int x, y, z;
        decode(g, n, x, y, z);
        const uint8_t c = cls[n];
        const bool bgk = (c == FLUID || c == BIO);
        const double rho = rho_in + (rho_out - rho_in) * (double)x / (double)(g.nx - 1);
        const float rb = bgk ? (float)(rho - 1.0) : 0.f;
#pragma unroll
        for (int i = 0; i < 19; ++i) f[i * g.N + s] = t19(i) * rb;
    }
}

// the flow's live sites: every class but bounce-back, NoDynamics only when
// some NoDynamics site touches a dynamic one (the class byte has no flags)
__device__ __forceinline__ bool flow_live(uint8_t cls, int nodyn_coupled) {
    return !(cls == BB || (cls == NODYN && !nodyn_coupled));
}

// need[n] = 1 when site n has no storage yet and streams, has a D3Q19
// neighbour that streams, or is given a nonzero population (nat, natural
// order, may be null)
__global__ void flow_need_kernel(Geo g, const uint8_t* cls, int nodyn_coupled, const int32_t* sidx,
                                 const float* nat, uint8_t* need) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        bool nd = false;
        if (sidx[n] < 0) {
            if (flow_live(cls[n], nodyn_coupled)) nd = true;
            else {
                int x, y, z;
                decode(g, n, x, y, z);
                const Site st = make_site(g, x, y, z, (uint32_t)n);
#pragma unroll
                for (int i = 1; i < 19; ++i)
                    if (st.inx(c19x(i)) && flow_live(cls[st.at(c19x(i), c19y(i), c19z(i))], nodyn_coupled)) nd = true;
            }
            if (!nd && nat)
                for (int i = 0; i < 19; ++i)
                    if (__float_as_uint(nat[i * g.N + n]) != 0u) nd = true;
        }
        need[n] = nd ? 1 : 0;
    }
}

// zero slots of storage indices [lo, hi): a site entering the storage holds
// what the full-lattice layout holds at a site nothing has written
__global__ void flow_zero_kernel(float* f, int64_t N, int64_t lo, int64_t hi) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t s = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < hi; s += stride)
#pragma unroll
        for (int i = 0; i < 19; ++i) f[i * N + s] = 0.f;
}

int flow_store_update(Ctx* c, const float* d_nat) {
    const int64_t N = c->geo.N;
    if (!c->d_fsidx) {
        int r = dalloc(c, &c->d_fsidx, (size_t)N);
        if (r) return r;
        CL_CUDA(cudaMemsetAsync(c->d_fsidx, 0xff, sizeof(int32_t) * N, c->stream));
        c->n_fstored = 0;
    }
    if (c->n_fstored == N) { c->fstore_dirty = false; return CL_OK; }
    uint8_t* need = reinterpret_cast<uint8_t*>(c->d_scratch);            // N bytes
    flow_need_kernel<<<grid_for(N, 256, 148 * 16), 256, 0, c->stream>>>(
        c->geo, c->d_ns_cls, c->flow_nodyn_coupled ? 1 : 0, c->d_fsidx, d_nat, need);
    CL_LAUNCH_CHECK("flow_need_kernel");
    int64_t first = 0, added = 0;
    int r = assign_storage(c, need, c->d_fsidx, nullptr, &c->n_fstored, &first, &added);
    if (r) return r;
    if (added > 0) {
        flow_zero_kernel<<<grid_for(added, 256, 148 * 16), 256, 0, c->stream>>>(c->d_f, N, first, first + added);
        CL_LAUNCH_CHECK("flow_zero_kernel");
    }
    c->fstore_dirty = false;
    return CL_OK;
}

__global__ void tracer_reset_kernel(FlowTracer* tr, double eps) {
    tr->count = 0; tr->head = 0; tr->converged = 0; tr->diverged = 0;
    tr->steps_done = 0; tr->converged_at = -1; tr->eps = eps; tr->last_energy = 0.0;
}

int flow_arm_tracer(Ctx* c, double eps) {
    tracer_reset_kernel<<<1, 1, 0, c->stream>>>(c->d_tracer, eps);
    CL_LAUNCH_CHECK("tracer_reset_kernel");
    return CL_OK;
}

int flow_init(Ctx* c) {
    // the storage starts afresh from the current classes
    if (c->d_fsidx) CL_CUDA(cudaMemsetAsync(c->d_fsidx, 0xff, sizeof(int32_t) * c->geo.N, c->stream));
    c->n_fstored = 0;
    int r = flow_store_update(c, nullptr);
    if (r) return r;
    flow_init_kernel<<<grid_for(c->geo.N, 256, 148 * 16), 256, 0, c->stream>>>(
        c->geo, c->d_f, c->d_fsidx, c->d_ns_cls, c->cfg.rho_in, c->cfg.rho_out);
    CL_LAUNCH_CHECK("flow_init_kernel");
    c->flow_parity = 0;
    return flow_arm_tracer(c, 0.0);
}

// One collideAndStream (two launches: the step, then the tracer update).
int flow_step(Ctx* c, int use_tracer) {
    if (c->fstore_dirty) { int r0 = flow_store_update(c, nullptr); if (r0) return r0; }
    if (c->flive_dirty) { int r0 = build_flow_list(c); if (r0) return r0; }
    FlowK k = make_flowk(c);
    k.list = c->d_flive;
    k.count = c->n_flive;
    if (!use_tracer) k.tracer = nullptr;
    // one wave: three 256-thread blocks (80 registers) per SM, each walking
    // the list grid-stride, so no block waits in a tail
    const int blocks = c->energy_blocks < 148 * 3 ? c->energy_blocks : 148 * 3;
    int r = timing_begin(c, CL_KERNEL_FLOW_STEP);
    if (r) return r;
    if (c->flow_parity == 0) flow_aa_kernel<0><<<blocks, 256, 0, c->stream>>>(k);
    else flow_aa_kernel<1><<<blocks, 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("flow_aa_kernel");
    if ((r = timing_end(c, CL_KERNEL_FLOW_STEP))) return r;
    c->launches += 2;
    const double inv = c->n_bgk > 0 ? 1.0 / (double)c->n_bgk : 0.0;
    flow_finalize_kernel<<<1, 512, 0, c->stream>>>(c->d_energy_part, blocks, inv, c->d_tracer, use_tracer);
    CL_LAUNCH_CHECK("flow_finalize_kernel");
    c->flow_parity ^= 1;
    return CL_OK;
}

// Density and momentum of every site from the current AA state
// (Palabos computeDensity / computeVelocity; IncBGK: velocity is j).
template <int PARITY>
__global__ void flow_macro_kernel(FlowK k, double* rho, float* u) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        const uint8_t cls = k.cls[n];
        float f[19];
        gather19_any<PARITY>(k, make_site(k.g, x, y, z, (uint32_t)n), f);
        float rb = 0.f, jx = 0.f, jy = 0.f, jz = 0.f;
        const bool bgk = (cls == FLUID || cls == BIO);
        if (bgk && x == 0) { rb = k.rb_in; regularize<-1>(f, rb, jx); }
        else if (bgk && x == k.g.nx - 1) { rb = k.rb_out; regularize<1>(f, rb, jx); }
        else {
#pragma unroll
            for (int i = 0; i < 19; ++i) {
                rb += f[i];
                jx += c19x(i) * f[i]; jy += c19y(i) * f[i]; jz += c19z(i) * f[i];
            }
            if (!bgk) { jx = jy = jz = 0.f; }
        }
        if (rho) rho[n] = 1.0 + (double)rb;
        if (u) { u[n] = jx; u[k.g.N + n] = jy; u[2 * k.g.N + n] = jz; }
    }
}

int flow_macro(Ctx* c, double* d_rho, float* d_u3, int) {
    if (!c->d_fsidx) { int r = flow_store_update(c, nullptr); if (r) return r; }
    FlowK k = make_flowk(c);
    const int blocks = grid_for(c->geo.N, 256, 148 * 16);
    if (c->flow_parity == 0) flow_macro_kernel<0><<<blocks, 256, 0, c->stream>>>(k, d_rho, d_u3);
    else flow_macro_kernel<1><<<blocks, 256, 0, c->stream>>>(k, d_rho, d_u3);
    CL_LAUNCH_CHECK("flow_macro_kernel");
    return CL_OK;
}

// Velocity statistics the reference takes after the flow solve for the
// Peclet calibration (complab.cpp:641-652): the sum of |u| and the maximum
// of u_x over x = 1..nx-2, the sum of u_x over the plane x = nx-2.  Fixed
// grid, per-block FP64 partials, one block adds them in index order.
template <int PARITY>
__global__ void flow_stats_kernel(FlowK k, double* part) {
    __shared__ double red[3][256];
    double su = 0.0, mx = -1.0 / 0.0, so = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t lo = k.g.plane, hi = k.g.N - k.g.plane;
    for (int64_t n = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < hi; n += stride) {
        int x, y, z;
        decode(k.g, n, x, y, z);
        const uint8_t cls = k.cls[n];
        float jx = 0.f, jy = 0.f, jz = 0.f;
        if (cls == FLUID || cls == BIO) {
            float f[19];
            gather19_any<PARITY>(k, make_site(k.g, x, y, z, (uint32_t)n), f);
#pragma unroll
            for (int i = 0; i < 19; ++i) { jx += c19x(i) * f[i]; jy += c19y(i) * f[i]; jz += c19z(i) * f[i]; }
        }
        su += sqrt((double)jx * jx + (double)jy * jy + (double)jz * jz);
        mx = fmax(mx, (double)jx);
        if (x == k.g.nx - 2) so += jx;
    }
    red[0][threadIdx.x] = su; red[1][threadIdx.x] = mx; red[2][threadIdx.x] = so;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            red[0][threadIdx.x] += red[0][threadIdx.x + o];
            red[1][threadIdx.x] = fmax(red[1][threadIdx.x], red[1][threadIdx.x + o]);
            red[2][threadIdx.x] += red[2][threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part[3 * blockIdx.x] = red[0][0]; part[3 * blockIdx.x + 1] = red[1][0]; part[3 * blockIdx.x + 2] = red[2][0]; }
}

__global__ void flow_stats_final(const double* part, int nb, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double su = 0.0, mx = -1.0 / 0.0, so = 0.0;
    for (int b = 0; b < nb; ++b) { su += part[3 * b]; mx = fmax(mx, part[3 * b + 1]); so += part[3 * b + 2]; }
    out[0] = su; out[1] = mx; out[2] = so;
}

int flow_stats(Ctx* c, double out[3]) {
    if (!c->d_fsidx) { int r = flow_store_update(c, nullptr); if (r) return r; }
    FlowK k = make_flowk(c);
    const int nb = 148 * 4;
    double* part = c->d_scratch;
    if (c->flow_parity == 0) flow_stats_kernel<0><<<nb, 256, 0, c->stream>>>(k, part);
    else flow_stats_kernel<1><<<nb, 256, 0, c->stream>>>(k, part);
    flow_stats_final<<<1, 32, 0, c->stream>>>(part, nb, part + 3 * nb);
    CL_LAUNCH_CHECK("flow_stats_kernel");
    CL_CUDA(cudaMemcpyAsync(out, part + 3 * nb, 3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

// sum of the velocity norm and count over the sites of one material in
// x = 1..nx-2: the masked computeAverage(*computeVelocityNorm(...), geometry,
// code) and MaskedScalarCounts3D of the reference's Peclet calibration
// (src/complab.cpp:625-640).  Bounce-back sites count with velocity zero.
template <int PARITY>
__global__ void flow_norm_masked_kernel(FlowK k, const uint8_t* mask, int code, double* part) {
    __shared__ double red[2][256];
    double su = 0.0, cnt = 0.0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t lo = k.g.plane, hi = k.g.N - k.g.plane;
    for (int64_t n = lo + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < hi; n += stride) {
        if (mask[n] != code) continue;
        cnt += 1.0;
        const uint8_t cls = k.cls[n];
        if (cls != FLUID && cls != BIO) continue;
        int x, y, z;
        decode(k.g, n, x, y, z);
        float f[19];
        gather19_any<PARITY>(k, make_site(k.g, x, y, z, (uint32_t)n), f);
        float jx = 0.f, jy = 0.f, jz = 0.f;
#pragma unroll
        for (int i = 0; i < 19; ++i) { jx += c19x(i) * f[i]; jy += c19y(i) * f[i]; jz += c19z(i) * f[i]; }
        su += sqrt((double)jx * jx + (double)jy * jy + (double)jz * jz);
    }
    red[0][threadIdx.x] = su; red[1][threadIdx.x] = cnt;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) { red[0][threadIdx.x] += red[0][threadIdx.x + o]; red[1][threadIdx.x] += red[1][threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = red[0][0]; part[2 * blockIdx.x + 1] = red[1][0]; }
}

__global__ void flow_norm_masked_final(const double* part, int nb, double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double su = 0.0, cnt = 0.0;
    for (int b = 0; b < nb; ++b) { su += part[2 * b]; cnt += part[2 * b + 1]; }
    out[0] = su; out[1] = cnt;
}

int flow_norm_masked(Ctx* c, int code, double out[2]) {
    if (!c->d_fsidx) { int r = flow_store_update(c, nullptr); if (r) return r; }
    FlowK k = make_flowk(c);
    const int nb = 148 * 4;
    double* part = c->d_scratch;
    if (c->flow_parity == 0) flow_norm_masked_kernel<0><<<nb, 256, 0, c->stream>>>(k, c->d_mask, code, part);
    else flow_norm_masked_kernel<1><<<nb, 256, 0, c->stream>>>(k, c->d_mask, code, part);
    flow_norm_masked_final<<<1, 32, 0, c->stream>>>(part, nb, part + 2 * nb);
    CL_LAUNCH_CHECK("flow_norm_masked_kernel");
    CL_CUDA(cudaMemcpyAsync(out, part + 2 * nb, 2 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

// natural-order copy of the populations (to_natural) or upload from natural
// order (requires parity 0 afterwards).
template <int PARITY>
__global__ void flow_io_kernel(FlowK k, float* nat, int to_natural) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < k.g.N; n += stride) {
        if (to_natural) {
            float f[19];
            gather19_any<PARITY>(k, site_of(k.g, n), f);
#pragma unroll
            for (int i = 0; i < 19; ++i) nat[i * k.g.N + n] = f[i];
        } else {
            // every site given a nonzero population is stored by now
            const int32_t s = k.sidx[n];
            if (s < 0) continue;
#pragma unroll
            for (int i = 0; i < 19; ++i) k.f[i * k.g.N + s] = nat[i * k.g.N + n];
        }
    }
}

int flow_population_io(Ctx* c, float* d_nat, int to_natural) {
    if (!to_natural || !c->d_fsidx) {
        int r = flow_store_update(c, to_natural ? nullptr : d_nat);
        if (r) return r;
    }
    FlowK k = make_flowk(c);
    const int blocks = grid_for(c->geo.N, 256, 148 * 16);
    if (!to_natural || c->flow_parity == 0) flow_io_kernel<0><<<blocks, 256, 0, c->stream>>>(k, d_nat, to_natural);
    else flow_io_kernel<1><<<blocks, 256, 0, c->stream>>>(k, d_nat, to_natural);
    CL_LAUNCH_CHECK("flow_io_kernel");
    if (!to_natural) c->flow_parity = 0;
    return CL_OK;
}

}  // namespace cl
