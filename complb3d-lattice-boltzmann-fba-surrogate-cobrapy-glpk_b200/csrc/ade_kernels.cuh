// ade_kernels.cuh -- fused multi-solute D3Q7 advection-diffusion-reaction step.
//
// One launch does, for every interior site and every mobile solute, what the
// reference does in separate whole-lattice passes (src/complab.cpp:1252-1374,
// 1849-1857): AdvectionDiffusionBGKdynamics collide, run_kinetics +
// update_rxnLattices, the dC reset + run_abiotic_kinetics /
// surfaceAbioticKinetics3D + update_abiotic_rxnLattices, run_equilibrium_biotic
// (Newton), and stream.  The increment lattices dC/dB of the reference
// (whole-lattice copies every step, complab.cpp:1264) never exist: increments
// stay in shared memory of the thread that owns the voxel.
//
// Per site the reaction chain only needs the solute densities, and every
// reference processor adds t_i*dC to the post-collision populations, so:
//   pass 1  gathers the populations and sums the densities,
//   chain   runs kinetics -> abiotic -> equilibrium on the densities (FP64),
//   pass 2  re-gathers (L1/L2 hit), collides, adds t_i*dC_total, streams.
// HBM traffic stays at one read and one write of 7 FP32 populations per
// solute; the FP64 Newton state never shares registers with the populations.
//
// Boundary planes x = 0 and x = nx-1 run in a second, small launch after the
// interior one: a zero-gradient face needs the pre-collision density of its
// neighbour plane, which the interior launch records (FlatAdiabaticBoundary-
// Functional3D sets the boundary density to that value after each stream).
//
// Dissolution (surfaceDissolutionKinetics3D) is the one processor that writes
// other voxels' increments.  A small launch before the fused one evaluates
// every phase voxel's release from the water of its open neighbours (their
// densities after this step's kinetics, recomputed there) and records it per
// phase voxel; the fused kernel then gathers, at each voxel flagged as next to
// a phase, its neighbours' records into the abiotic increment, in the order
// the reference's serial scatter adds them.
#pragma once
#include "internal.h"
#include "newton.cuh"

namespace cl {

#define THRD 1e-12
constexpr int kGroup = 4;   // solutes whose populations are in flight together

struct AdeK {
    Geo g;
    float* pop;               // n_mob * 7 * N
    const uint8_t* cls;
    const float* u;           // 3*N
    double* imm;              // S*N
    double* bio;              // M*N
    float* rho_adj;           // n_mob * 2 * plane
    int32_t* eq_iters;        // N (may be null)
    double* eq_x;             // NC*N previous solutions (null: cold start only)
    const uint8_t* mask;      // N material numbers
    const uint8_t* phase;     // N phase ids (null without dissolution)
    double* rel;              // S*N releases of the phase voxels (null without dissolution)
    unsigned long long* counters;
    int nodyn_coupled;
    int parity;
    AdeParams p;
    EqDev e;
};

template <int PARITY>
__device__ __forceinline__ void gather7(const float* pop, uint32_t N, const Site& st, float* f) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        if (PARITY == 0 || !st.inx(-c7x(i))) f[i] = pop[i * N + st.n];
        else f[i] = pop[opp7(i) * N + st.at(-c7x(i), -c7y(i), -c7z(i))];
    }
}

template <int PARITY>
__device__ __forceinline__ void scatter7(float* pop, uint32_t N, const Site& st, const float* f) {
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        if (PARITY == 0 || !st.inx(c7x(i))) pop[opp7(i) * N + st.n] = f[i];
        else pop[i * N + st.at(c7x(i), c7y(i), c7z(i))] = f[i];
    }
}

// AdvectionDiffusionBGKdynamics: geq_i = t_i rho (1 + c_i.u / cs2), cs2 = 1/4
__device__ __forceinline__ void collide7(float* f, float om, float ux, float uy, float uz, float& rho) {
    float r = 0.f;
#pragma unroll
    for (int i = 0; i < 7; ++i) r += f[i];
    rho = r;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        const float cu = c7x(i) * ux + c7y(i) * uy + c7z(i) * uz;
        const float geq = t7(i) * r * (1.f + 4.f * cu);
        f[i] = f[i] - om * (f[i] - geq);
    }
}

// Table-driven rate law (defineRxnKinetics / defineAbioticRxnKinetics ABI).
// C is a column with stride cs; R, B, BR columns with stride bd.
// Concentrations below thrd read as zero, as the processors floor them
// before the call.
static __device__ void rates_dev(const AdeParams& p, int abiotic, const double* C, int cs, const double* B,
                          double* R, double* BR, int bd) {
    for (int s = 0; s < p.S; ++s) R[s * bd] = 0.0;
    if (!abiotic) for (int m = 0; m < p.M; ++m) BR[m * bd] = 0.0;
    for (int k = 0; k < p.n_rxn; ++k) {
        const cl_rxn& r = p.rxn[k];
        if ((r.microbe < 0) != (abiotic != 0)) continue;
        double rate = r.k;
        if (r.microbe >= 0) {
            const double b = B[r.microbe * bd];
            if (!(b > 0.0)) continue;
            rate *= b;
        }
        for (int j = 0; j < r.n_monod; ++j) {
            const double c0 = C[r.monod_s[j] * cs];
            const double c = c0 < THRD ? 0.0 : c0;
            rate *= c / (r.monod_ks[j] + c);
        }
        for (int j = 0; j < r.n_mass; ++j) {
            const double c0 = C[r.mass_s[j] * cs];
            rate *= c0 < THRD ? 0.0 : c0;
        }
        for (int s = 0; s < p.S; ++s) R[s * bd] = fma(r.nu[s], rate, R[s * bd]);
        if (!abiotic) BR[r.microbe * bd] = fma(r.yield, rate, BR[r.microbe * bd]);
    }
    if (!abiotic)
        for (int m = 0; m < p.M; ++m) BR[m * bd] -= p.decay[m] * fmax(B[m * bd], 0.0);
    for (int s = 0; s < p.S; ++s) if (!isfinite(R[s * bd])) R[s * bd] = 0.0;
    if (!abiotic) for (int m = 0; m < p.M; ++m) if (!isfinite(BR[m * bd])) BR[m * bd] = 0.0;
}

// Surrogate reaction type of one voxel (run_surrogate3D,
// src/complab3d_processors_surrogate.hh:94-295).  Reads the densities the
// kinetics read (before update_rxnLattices), adds its thresholded increments
// into D (solutes) and DB (biomass), which the caller applies together with
// the kinetics increments, as the shared dC/dB lattices of the reference do.
static __device__ __noinline__ void surrogate_chain(const AdeParams& p, const double* Cur, int cs, const double* B,
                                             double* D, double* DB, int bd) {
    double conc[CL_MAX_SOLUTES], draw[CL_MAX_SOLUTES];
    bool any = false;
    for (int o = 0; o < p.n_srg; ++o) any = any || B[p.srg[o].microbe * bd] > THRD;
    if (!any) return;
    for (int s = 0; s < p.S; ++s) {
        const double c = Cur[s * cs];
        conc[s] = c > THRD ? c : 0.0;
        draw[s] = 0.0;
    }
    for (int o = 0; o < p.n_srg; ++o) {
        const cl_srg_organism& org = p.srg[o];
        const SrgNetDev& net = p.net[org.net];
        const double b = B[org.microbe * bd];
        if (!(b > THRD)) continue;
        // Michaelis-Menten uptake estimates, capped by the exhaustion flux
        // (MetabolicConfig::exhaustionFlux, complab3d_metabolic.hh:504-519)
        double fin[CL_MAX_SOLUTES];
        const double denom = b * org.mw * p.dt;
        for (int s = 0; s < p.S; ++s) {
            const double av = conc[s];
            const double mm = (org.kc[s] + av > 0.0) ? av / (org.kc[s] + av) : 0.0;
            double exh = 0.0;
            if (denom > 1e-30) { exh = -av * 3.6e6 / denom; if (exh < -1e4) exh = -1e4; }
            double v = org.vmax[s] > THRD ? org.vmax[s] * mm : -exh * mm;
            const double cap = -exh;
            if (cap > 0.0 && v > cap) v = cap;
            fin[s] = v;
        }
        // the network: mapminmax inputs, tanh hidden layers, linear output
        float a[CL_SRG_MAX_WIDTH], t[CL_SRG_MAX_WIDTH];
        const int win = net.w[0];
        for (int i = 0; i < win; ++i) {
            const int kind = org.in_kind[i], idx = org.in_index[i];
            float v = kind == CL_SRG_IN_FIN ? (float)fin[idx] : kind == CL_SRG_IN_CONC ? (float)conc[idx] : (float)b;
            v = fminf(fmaxf(v, net.xlo[i]), net.xhi[i]);
            a[i] = (v - net.xo[i]) * net.xg[i] + net.xymin;
        }
        for (int l = 0; l < net.L; ++l) {
            const int wi = net.w[l], wo = net.w[l + 1];
            const float* W = net.params + net.poff[l];
            for (int q = 0; q < wo; ++q) {
                float acc = __ldg(W + wo * wi + q);
                for (int i = 0; i < wi; ++i) acc = fmaf(__ldg(W + q * wi + i), a[i], acc);
                t[q] = (l < net.L - 1) ? tanhf(acc) : acc;
            }
            for (int q = 0; q < wo; ++q) a[q] = t[q];
        }
        double mu = 0.0;
        double fout[CL_MAX_SOLUTES];
        for (int s = 0; s < p.S; ++s) fout[s] = fin[s];
        for (int q = 0; q < net.w[net.L]; ++q) {
            const double y = ((double)a[q] - net.yymin) / net.yg[q] + net.yo[q];
            if (org.out_kind[q] == CL_SRG_OUT_GROWTH) mu = y;
            else fout[org.out_index[q]] = y;
        }
        if (mu < 1e-8 || !isfinite(mu)) mu = 0.0;     // the exported model's dust / NaN guard
        // growthToDeltaB / decayToDeltaB (complab3d_metabolic.hh:487-500)
        double dB = (fabs(mu) < THRD) ? -org.kd * b * p.dt : mu * b * p.dt / 3600.0;
        if (dB + b < 0.0) dB = -b;
        if (fabs(dB) > THRD) DB[org.microbe * bd] += dB;
        // fluxToDeltaC: positive Fout is consumed
        for (int s = 0; s < p.S; ++s) draw[s] += -fout[s] * b * org.mw * p.dt / 3.6e6;
    }
    for (int s = 0; s < p.S; ++s) {
        double d = draw[s];
        if (fabs(d) <= THRD) continue;
        if (d + conc[s] < 0.0) d = -conc[s];
        if (d > 0.0) d = 0.0;
        if (fabs(d) > THRD) D[s * bd] += d;
    }
}

// run_kinetics (part1.hh:63-146) and run_surrogate3D deposit into the same
// dC/dB lattices, each contribution only if above thrd: the increments of one
// voxel into R (solutes) and BR (biomass), B its floored biomass.  Not applied.
__device__ __forceinline__ void kinetics_increments(const AdeParams& p, const double* bio, int64_t N, int64_t n,
                                                    const double* Cur, int cs, double* R, double* B, double* BR,
                                                    int bd) {
    for (int m = 0; m < p.M; ++m) { const double b = bio[m * N + n]; B[m * bd] = b < THRD ? 0.0 : b; }
    if (p.do_kin) {
        rates_dev(p, 0, Cur, cs, B, R, BR, bd);
        for (int s = 0; s < p.S; ++s) {
            const double d = R[s * bd] * p.dt;
            R[s * bd] = (d > THRD || d < -THRD) ? d : 0.0;
        }
        for (int m = 0; m < p.M; ++m) {
            const double d = BR[m * bd] * p.dt;
            BR[m * bd] = (d > THRD || d < -THRD) ? d : 0.0;
        }
    } else {
        for (int s = 0; s < p.S; ++s) R[s * bd] = 0.0;
        for (int m = 0; m < p.M; ++m) BR[m * bd] = 0.0;
    }
    if (p.n_srg > 0) surrogate_chain(p, Cur, cs, B, R, BR, bd);
}

// The dissolution increments that reach voxel n (surfaceDissolutionKinetics3D,
// dissolutionVOP.hh:392-425): the products of each face neighbour that carries
// a phase, and the voxel's own mineral decrement.  Neighbours are visited in
// increasing site order with the voxel itself between -z and +z, the order in
// which the reference's serial scatter adds into this voxel's dC.
__device__ __forceinline__ void dissol_gather(const AdeK& k, int64_t n, int x, int y, int z, uint8_t cls,
                                              double* D, int bd) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane, nz = k.g.nz;
    const int64_t q[7] = {n - plane, n - nz, n - 1, n, n + 1, n + nz, n + plane};
    const bool ok[7] = {x - 1 >= 1, y > 0, z > 0, (cls & F_PHASE_SELF) != 0,
                        z < k.g.nz - 1, y < k.g.ny - 1, x + 1 <= k.g.nx - 2};
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        if (!ok[j]) continue;
        const int pid = k.phase[q[j]];
        if (pid == 0) continue;
        const int sM = p.phase[pid - 1].substrate;
        if (j == 3) { D[sM * bd] += k.rel[(int64_t)sM * N + n]; continue; }
        for (int s = 0; s < p.S; ++s)
            if (s != sM) D[s * bd] += k.rel[(int64_t)s * N + q[j]];
    }
}

// The reaction chain of one voxel.  Cur holds the current densities (updated
// as each processor applies its increments), App the total increment per
// solute.  Returns 1 if the equilibrium solve did not converge.
template <int NC>
__device__ int reaction_chain(const AdeK& k, int64_t n, int x, int y, int z, uint8_t cls, double* Cur, double* App,
                              int cs, double* R, double* B, double* BR, int bd) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N;
    int nonconv = 0;
    // kinetics and surrogate increments; update_rxnLattices (:338-429) applies
    // the sums that exceed thrd
    if (p.do_kin || p.n_srg > 0) {
        kinetics_increments(p, k.bio, N, n, Cur, cs, R, B, BR, bd);
        for (int s = 0; s < p.S; ++s) {
            const double d = R[s * bd];
            if (d > THRD || d < -THRD) { Cur[s * cs] += d; App[s * cs] += d; }
        }
        for (int m = 0; m < p.M; ++m) {
            const double d = BR[m * bd];
            if (d > THRD || d < -THRD) k.bio[m * N + n] += d;
        }
    }
    // dC = dC0; run_abiotic_kinetics | surfaceAbioticKinetics3D (thresholded);
    // + surfaceDissolutionKinetics3D; update_abiotic_rxnLattices applies the
    // sums that exceed thrd
    const bool abio = p.do_abio && (!p.surface_only || (cls & F_SURFACE));
    const bool dis = p.do_dissol && (cls & (F_PHASE_NBR | F_PHASE_SELF));
    if (abio || dis) {
        if (abio) {
            rates_dev(p, 1, Cur, cs, nullptr, R, nullptr, bd);
            for (int s = 0; s < p.S; ++s) {
                const double d = R[s * bd] * p.dt;
                R[s * bd] = (d > THRD || d < -THRD) ? d : 0.0;
            }
        } else {
            for (int s = 0; s < p.S; ++s) R[s * bd] = 0.0;
        }
        if (dis) dissol_gather(k, n, x, y, z, cls, R, bd);
        for (int s = 0; s < p.S; ++s) {
            const double d = R[s * bd];
            if (d > THRD || d < -THRD) { Cur[s * cs] += d; App[s * cs] += d; }
        }
    }
    // run_equilibrium_biotic (part4_eqsolver.hh:1355-1494): species floored at
    // 1e-30; Newton applied only when converged (run_equilibrium_NR, NR_reserve.hh:734)
    if constexpr (NC > 0) {
        const EqDev& e = k.e;
        double x[NC], T[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = 0.0;
        for (int i = 0; i < e.ns; ++i) {
            if (!e.active[i]) continue;
            const double c = fmin(fmax(Cur[i * cs], 1e-30), 10.0);
#pragma unroll
            for (int j = 0; j < NC; ++j) T[j] = fma(e.stoich[i][j], c, T[j]);
        }
        auto cold = [&](double* xs) {
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                double c = 1e-7;
                const int idx = e.comp_species[j];
                if (idx >= 0) c = Cur[idx * cs];
                xs[j] = log10(fmin(fmax(c, 1e-30), 10.0));
            }
        };
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = fmax(T[j], 1e-30);
        int conv = 0, it = 0;
        bool warm = false;
        if (k.eq_x) {
            warm = true;
#pragma unroll
            for (int j = 0; j < NC; ++j) { x[j] = k.eq_x[(int64_t)j * N + n]; warm = warm && (x[j] == x[j]); }
        }
        // the warm attempt (previous solution, warm_iter iterations), then the
        // cold start; one call site keeps one copy of the solver in the kernel
        for (int phase = warm ? 0 : 1; phase < 2; ++phase) {
            if (phase == 1) cold(x);
            it += eq_newton<NC>(e, T, x, phase == 0 ? p.eq.warm_iter : p.eq.max_iter, p.eq.tol, &conv);
            if (conv) break;
        }
        if (k.eq_x && conv) {
#pragma unroll
            for (int j = 0; j < NC; ++j) k.eq_x[(int64_t)j * N + n] = x[j];
        }
        if (k.eq_iters) k.eq_iters[n] = it;
        if (!conv) nonconv = 1;
        else {
            for (int s = 0; s < p.S && s < e.ns; ++s) {
                const double conc = fmax(Cur[s * cs], 1e-30);
                double eqc = e.active[s] ? species_c<NC>(e, s, x) : fmin(conc, 10.0);
                eqc = fmin(fmax(eqc, 1e-30), 10.0);
                double d = eqc - conc;
                const double mx = fmax(1e-9, 0.1 * fabs(conc));
                if (fabs(d) > mx) d = d > 0 ? mx : -mx;
                if (conc + d < 1e-20) d = 1e-20 - conc;
                if (fabs(d) > THRD) { Cur[s * cs] += d; App[s * cs] += d; }
            }
        }
    }
    return nonconv;
}

// A tile of kTile = 2 x kBlock sites of whole z-rows is one block iteration;
// each thread owns two sites of it.  Only the reactive sites (about the
// porosity's share) run the reaction chain, so after pass 1 the block
// compacts them into a list and its threads work through that list, each on
// the shared-memory columns of the site it took and on its own scratch
// columns: the FP64 chain then runs on full warps, and a tile of two sites
// per thread keeps about two thirds of the block busy in it.
constexpr int kBlock = 256;
constexpr int kSitesPerThread = 2;
constexpr int kTile = kBlock * kSitesPerThread;

// virtual thread v of a tile -> (row offset, z, stride) as RowMap does for threads
struct TileMap {
    int rpb, zstep;
    __device__ __forceinline__ void at(int nz, int v, int& lrow, int& z0, bool& active) const {
        if (nz >= kTile) { lrow = 0; z0 = v; active = true; }
        else { lrow = v / nz; z0 = v - lrow * nz; active = lrow < rpb; }
    }
};

__device__ __forceinline__ TileMap make_tilemap(int nz) {
    TileMap m;
    if (nz >= kTile) { m.rpb = 1; m.zstep = kTile; }
    else { m.rpb = kTile / nz; m.zstep = nz; }
    return m;
}

template <int NMOB, int NC, int PARITY>
__global__ void __launch_bounds__(kBlock, 2) ade_main_kernel(const __grid_constant__ AdeK k) {
    extern __shared__ double sm[];
    __shared__ uint32_t s_n[kTile];        // site of each tile column
    __shared__ int s_xyz[kTile][3];
    __shared__ uint8_t s_cls[kTile];
    __shared__ short s_list[kTile];        // compacted reactive columns
    __shared__ int s_count;
    const int t = threadIdx.x;
    const AdeParams& p = k.p;
    const int Mw = p.M > 0 ? p.M : 1;
    double* CurT = sm;                       // [S][kTile] densities of the tile's sites
    double* AppT = CurT + p.S * kTile;       // [S][kTile] their total increments
    double* Rw = AppT + p.S * kTile;         // [S][kBlock] per-thread scratch
    double* Bw = Rw + p.S * kBlock;          // [M][kBlock]
    double* BRw = Bw + Mw * kBlock;          // [M][kBlock]
    const int64_t N = k.g.N, plane = k.g.plane;
    const uint32_t N32 = (uint32_t)N;
    const bool any_rxn = p.do_kin || p.do_abio || p.n_srg > 0 || p.do_dissol || NC > 0;
    unsigned long long nonconv = 0;
    const TileMap tm = make_tilemap(k.g.nz);
    const int row_lo = k.g.ny, row_hi = (k.g.nx - 1) * k.g.ny;     // interior x = 1 .. nx-2
    // every thread of a block runs the same iterations (the barriers below)
    for (int row0 = row_lo + blockIdx.x * tm.rpb; row0 < row_hi; row0 += gridDim.x * tm.rpb) {
      for (int zb = 0; zb < k.g.nz; zb += tm.zstep) {
        // the tile's sites: live (streams) and reactive masks, site data in shared memory
        unsigned lvm = 0, rcm = 0;
#pragma unroll
        for (int j = 0; j < kSitesPerThread; ++j) {
            const int v = t + j * kBlock;
            int lrow, z0; bool act;
            tm.at(k.g.nz, v, lrow, z0, act);
            const int row = row0 + lrow, z = zb + z0;
            if (!(act && row < row_hi && z < k.g.nz)) continue;
            const int x = row / k.g.ny, y = row - x * k.g.ny;
            const uint32_t n = (uint32_t)row * (uint32_t)k.g.nz + (uint32_t)z;
            const uint8_t cls = k.cls[n];
            const uint8_t dyn = cls & 3;
            // bounce-back sites are a no-op of the AA step, unless their mask
            // reopened to pore: then they react (the processors test the mask)
            if ((dyn == BB && !(cls & F_REACTIVE)) || (dyn == NODYN && !k.nodyn_coupled)) continue;
            lvm |= 1u << j;
            // the processors test the mask, not the dynamics: a NoDynamics
            // site whose mask reopened to pore reacts too
            if (any_rxn && (cls & F_REACTIVE)) rcm |= 1u << j;
            s_n[v] = n; s_xyz[v][0] = x; s_xyz[v][1] = y; s_xyz[v][2] = z; s_cls[v] = cls;
        }
        if (any_rxn) {
            // pass 1: the populations of a group of solutes in flight at once, then the densities
#pragma unroll 1
            for (int j = 0; j < kSitesPerThread; ++j) {
                if (!((rcm >> j) & 1u)) continue;
                const int v = t + j * kBlock;
                const uint32_t n = s_n[v];
                const Site st = make_site(k.g, s_xyz[v][0], s_xyz[v][1], s_xyz[v][2], n);
                for (int s = 0; s < p.S; ++s) AppT[s * kTile + v] = 0.0;
#pragma unroll
                for (int m0 = 0; m0 < NMOB; m0 += kGroup) {
                    float f[kGroup][7];
#pragma unroll
                    for (int q = 0; q < kGroup; ++q)
                        if (m0 + q < NMOB) gather7<PARITY>(k.pop + (int64_t)(m0 + q) * 7 * N, N32, st, f[q]);
#pragma unroll
                    for (int q = 0; q < kGroup; ++q) {
                        if (m0 + q >= NMOB) continue;
                        float r = 0.f;
#pragma unroll
                        for (int i = 0; i < 7; ++i) r += f[q][i];
                        CurT[p.mob_index[m0 + q] * kTile + v] = (double)r;
                    }
                }
                for (int s = 0; s < p.S; ++s)
                    if (p.mob_slot[s] < 0) CurT[s * kTile + v] = k.imm[(int64_t)s * N + n];
            }
            if (t == 0) s_count = 0;
            __syncthreads();
            // compact the reactive columns (warp-aggregated slots)
#pragma unroll
            for (int j = 0; j < kSitesPerThread; ++j) {
                const bool rc = (rcm >> j) & 1u;
                const unsigned ball = __ballot_sync(0xffffffffu, rc);
                int base = 0;
                if ((t & 31) == 0 && ball) base = atomicAdd(&s_count, __popc(ball));
                base = __shfl_sync(0xffffffffu, base, 0);
                if (rc) s_list[base + __popc(ball & ((1u << (t & 31)) - 1u))] = (short)(t + j * kBlock);
            }
            __syncthreads();
            const int cnt = s_count;
            for (int r = t; r < cnt; r += kBlock) {
                const int c = s_list[r];
                double* cCur = CurT + c;
                double* cApp = AppT + c;
                const uint32_t cn = s_n[c];
                nonconv += reaction_chain<NC>(k, cn, s_xyz[c][0], s_xyz[c][1], s_xyz[c][2], s_cls[c],
                                              cCur, cApp, kTile, Rw + t, Bw + t, BRw + t, kBlock);
                for (int s = 0; s < p.S; ++s)
                    if (p.mob_slot[s] < 0 && cApp[s * kTile] != 0.0) k.imm[(int64_t)s * N + cn] += cApp[s * kTile];
            }
            __syncthreads();
        }
        // keep the second gather after the chain: hoisting it would hold all
        // populations in registers across the Newton solve
        asm volatile("" ::: "memory");
        // pass 2: gather every solute (L1/L2 hits after pass 1), collide, add t_i*dC, stream
#pragma unroll 1
        for (int j = 0; j < kSitesPerThread; ++j) {
            if (!((lvm >> j) & 1u)) continue;
            const int v = t + j * kBlock;
            const bool rc = (rcm >> j) & 1u;
            const uint32_t n = s_n[v];
            const int x = s_xyz[v][0];
            const uint8_t dyn = s_cls[v] & 3;
            const Site st = make_site(k.g, x, s_xyz[v][1], s_xyz[v][2], n);
            const float ux = k.u[n], uy = k.u[N + n], uz = k.u[2 * N + n];
            const bool adj = (x == 1 || x == k.g.nx - 2);
#pragma unroll
            for (int m0 = 0; m0 < NMOB; m0 += kGroup) {
                float f[kGroup][7];
#pragma unroll
                for (int q = 0; q < kGroup; ++q)
                    if (m0 + q < NMOB) gather7<PARITY>(k.pop + (int64_t)(m0 + q) * 7 * N, N32, st, f[q]);
#pragma unroll
                for (int q = 0; q < kGroup; ++q) {
                    const int m = m0 + q;
                    if (m >= NMOB) continue;
                    float rho = 0.f;
                    if (dyn == BB) {
                        // BounceBack's collision swaps opposite populations; in the
                        // AA layout swap + scatter leaves every slot as it was, so
                        // only the reaction increment moves anything
#pragma unroll
                        for (int i = 1; i < 4; ++i) { const float tmp = f[q][i]; f[q][i] = f[q][i + 3]; f[q][i + 3] = tmp; }
                    } else if (dyn != NODYN) {
                        const float om = (dyn == BIO) ? p.omega_bio[m] : p.omega_pore[m];
                        collide7(f[q], om, ux, uy, uz, rho);
                    } else if (adj) {
#pragma unroll
                        for (int i = 0; i < 7; ++i) rho += f[q][i];
                    }
                    const float d = rc ? (float)AppT[p.mob_index[m] * kTile + v] : 0.f;
                    if (d != 0.f) {
#pragma unroll
                        for (int i = 0; i < 7; ++i) f[q][i] += t7(i) * d;
                    }
                    if (adj && dyn != BB) {
                        const int side = (x == 1) ? 0 : 1;
                        k.rho_adj[((int64_t)m * 2 + side) * plane + (n - (int64_t)x * plane)] = rho;
                    }
                }
#pragma unroll
                for (int q = 0; q < kGroup; ++q)
                    if (m0 + q < NMOB) scatter7<PARITY>(k.pop + (int64_t)(m0 + q) * 7 * N, N32, st, f[q]);
            }
        }
        // no barrier needed before the next tile: after the chain's barrier
        // every thread reads only its own columns
      }
    }
    if (nonconv) atomicAdd(&k.counters[0], nonconv);
}

// x = 0 and x = nx-1: AdvectionDiffusionBoundaryDynamics (the one unknown
// population = prescribed density - the six known ones) then BGK collide.
template <int NMOB, int PARITY>
__global__ void __launch_bounds__(256) ade_boundary_kernel(const __grid_constant__ AdeK k) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < 2 * plane; q += stride) {
        const int side = q >= plane ? 1 : 0;
        const int64_t p2 = q - side * plane;
        const int64_t n = side ? (N - plane + p2) : p2;
        const uint8_t dyn = k.cls[n] & 3;
        if (dyn == BB) continue;
        if (dyn == NODYN && !k.nodyn_coupled) continue;
        int x, y, z;
        decode(k.g, n, x, y, z);
        const Site st = make_site(k.g, x, y, z, (uint32_t)n);
        const float ux = k.u[n], uy = k.u[N + n], uz = k.u[2 * N + n];
#pragma unroll
        for (int m = 0; m < NMOB; ++m) {
            float* pm = k.pop + (int64_t)m * 7 * N;
            float f[7];
            gather7<PARITY>(pm, (uint32_t)N, st, f);
            if (dyn != NODYN) {
                const int unk = side == 0 ? 4 : 1;
                const int neu = side == 0 ? p.left_neu[m] : p.right_neu[m];
                const float rb = neu ? k.rho_adj[((int64_t)m * 2 + side) * plane + p2]
                                     : (side == 0 ? p.left_val[m] : p.right_val[m]);
                float s = 0.f;
#pragma unroll
                for (int i = 0; i < 7; ++i) if (i != unk) s += f[i];
                f[unk] = rb - s;
                const float om = (dyn == BIO) ? p.omega_bio[m] : p.omega_pore[m];
                float rho;
                collide7(f, om, ux, uy, uz, rho);
            }
            scatter7<PARITY>(pm, (uint32_t)N, st, f);
        }
    }
}

inline AdeK make_adek(Ctx* c) {
    AdeK k;
    k.g = c->geo;
    k.pop = c->d_g;
    k.cls = c->d_ade_cls;
    k.u = c->d_u;
    k.imm = c->d_imm;
    k.bio = c->d_bio;
    k.rho_adj = c->d_rho_adj;
    k.eq_iters = c->d_eq_iters;
    k.eq_x = c->d_eq_x;
    k.mask = c->d_mask;
    k.phase = c->d_phase;
    k.rel = c->d_rel;
    k.counters = c->d_counters;
    k.nodyn_coupled = c->ade_nodyn_coupled ? 1 : 0;
    k.parity = c->ade_parity;
    k.p = c->ap;
    eqdev_from_system(c->cfg.eq, k.e);
    return k;
}

// the phase voxels' releases of this step (dissolution.cu), before the fused launch
int dissol_release(Ctx* c, const AdeK& k);

template <int NMOB, int NC>
inline int launch_step(Ctx* c, const AdeK& k) {
    const int bd = kBlock;
    const int S = c->ap.S, M = c->ap.M > 0 ? c->ap.M : 1;
    const bool any_rxn = c->ap.do_kin || c->ap.do_abio || c->ap.n_srg > 0 || c->ap.do_dissol || NC > 0;
    const size_t smem = any_rxn ? ((size_t)2 * S * kTile + (size_t)(S + 2 * M) * kBlock) * sizeof(double) : 0;
    const int64_t interior = c->geo.N - 2 * c->geo.plane;
    const int blocks = grid_for(interior, bd, 148 * 8);
    int r = CL_OK;
    if (c->ap.do_dissol && (r = dissol_release(c, k))) return r;
    if ((r = timing_begin(c, CL_KERNEL_ADE_MAIN))) return r;
    if (c->ade_parity == 0) {
        auto kern = ade_main_kernel<NMOB, NC, 0>;
        CL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<blocks, bd, smem, c->stream>>>(k);
    } else {
        auto kern = ade_main_kernel<NMOB, NC, 1>;
        CL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<blocks, bd, smem, c->stream>>>(k);
    }
    CL_LAUNCH_CHECK("ade_main_kernel");
    if ((r = timing_end(c, CL_KERNEL_ADE_MAIN))) return r;
    c->launches += 2;
    const int bblocks = grid_for(2 * c->geo.plane, bd, 148 * 4);
    if (c->ade_parity == 0) ade_boundary_kernel<NMOB, 0><<<bblocks, bd, 0, c->stream>>>(k);
    else ade_boundary_kernel<NMOB, 1><<<bblocks, bd, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("ade_boundary_kernel");
    c->ade_parity ^= 1;
    return CL_OK;
}

// one translation unit per component count instantiates these
int ade_step_nc0(Ctx* c); int ade_step_nc1(Ctx* c); int ade_step_nc2(Ctx* c);
int ade_step_nc3(Ctx* c); int ade_step_nc4(Ctx* c); int ade_step_nc5(Ctx* c);

}  // namespace cl
