// ade_kernels.cuh -- the multi-solute D3Q7 advection-diffusion-reaction step.
//
// One step does, for every interior site and every mobile solute, what the
// reference does in separate whole-lattice passes (src/complab.cpp:1252-1374,
// 1849-1857): AdvectionDiffusionBGKdynamics collide, run_kinetics +
// update_rxnLattices, the dC reset + run_abiotic_kinetics /
// surfaceAbioticKinetics3D + update_abiotic_rxnLattices, run_equilibrium_biotic
// (Newton), and stream.  The increment lattices dC/dB of the reference
// (whole-lattice copies every step, complab.cpp:1264) never exist.
//
// Per site the reaction chain only needs the solute densities, and every
// reference processor adds t_i*dC to the post-collision populations; the BGK
// collision keeps each density, so the chain can run on the pre-collision
// densities before the streaming launch:
//   ade_react_kernel   one thread per reactive site (the live list): gathers
//                      the populations, sums the densities, runs kinetics ->
//                      abiotic (+ dissolution) -> equilibrium in FP64, writes
//                      the total increment of each mobile solute to dc;
//   ade_stream_kernel  one thread per live site (the live list): gathers, collides, adds
//                      t_i*dc, streams (AA pattern, in place).
// The interior is cut into slabs of x planes: slab j streams while slab j+1
// reacts, on two streams.
//
// Boundary planes x = 0 and x = nx-1 run in a third, small launch: a
// zero-gradient face needs the pre-collision density of its neighbour plane,
// which the streaming launch records (FlatAdiabaticBoundaryFunctional3D sets
// the boundary density to that value after each stream).
//
// Dissolution (surfaceDissolutionKinetics3D) is the one processor that writes
// other voxels' increments.  A small launch before the reactions evaluates
// every phase voxel's release from the water of its open neighbours (their
// densities after this step's kinetics, recomputed there) and records it per
// phase voxel; the reaction chain then gathers, at each voxel flagged as next
// to a phase, its neighbours' records into the abiotic increment, in the order
// the reference's serial scatter adds them.
#pragma once
#include "internal.h"
#include "newton.cuh"
#include "pcf.cuh"

namespace cl {

#define THRD 1e-12
constexpr int kGroup = 4;        // solutes whose populations are in flight together (reactions)
constexpr int kStreamGroupEven = 4, kStreamGroupOdd = 4;
// the same in the streaming launch: an odd step's loads and stores address
// neighbours' slots, so fewer solutes are in flight there to stay within the
// 128 registers of two 256-thread blocks per SM
template <int PARITY> constexpr int stream_group() { return PARITY ? kStreamGroupOdd : kStreamGroupEven; }

struct AdeK {
    Geo g;
    float* pop;               // n_mob * 7 * N
    const uint8_t* cls;
    const float* u;           // 3*N
    double* imm;              // S*N
    double* bio;              // M*N
    float* rho_adj;           // n_mob * 2 * plane
    int32_t* eq_iters;        // N (may be null)
    // NC*N previous solutions and the ones before those, by storage index
    // (null: cold start only); FP32: a start needs no more, and transport
    // moves nearly every voxel's totals by more than the 1e-10 tolerance each
    // step, so a solve almost never stops at its start anyway (on the coupled
    // workload a few voxels in 1e5 per step)
    float* eq_x;
    float* eq_xp;
    const uint8_t* mask;      // N material numbers
    const uint8_t* phase;     // N phase ids (null without dissolution)
    double* rel;              // S*N releases of the phase voxels (null without dissolution)
    unsigned long long* counters;   // [0] non-converged solves, [1] sites without the storage they need
    const int32_t* sidx;            // N storage index of each site's slots
    // learned warm start (one-launch step only): network weights when trained,
    // and the ring the converged pairs of the sampled voxels go to
    const float* learn_w;
    const float* learn_norm;
    double* pair_T;
    double* pair_X;
    unsigned long long* pair_count;
    int64_t pair_cap;
    uint32_t pair_salt, pair_mask;
    int nodyn_coupled;
    int parity;
    AdeParams p;
    EqDev e;
};

// A site's slots in the compact storage: its own storage index and those of
// its six face neighbours (the sites at +c_d, d = 1..6); where x leaves the
// lattice the own index stands in (that slot is reflected, never read there).
// Returns false, with in-bounds substitutes, if a slot the step needs has no
// storage (the caller counts it; the step then reports an error).  An even
// step touches only the site's own slots: PARITY 0 looks up no neighbour.
struct SSite {
    uint32_t s;
    uint32_t nb[6];
    bool hxm, hxp;
    __device__ __forceinline__ bool inx(int dx) const { return dx < 0 ? hxm : (dx > 0 ? hxp : true); }
};

template <int PARITY = 1>
__device__ __forceinline__ bool make_ssite(const Geo& g, const int32_t* __restrict__ sidx, int x, int y, int z,
                                           uint32_t n, SSite& t) {
    const Site st = make_site(g, x, y, z, n);
    bool ok = true;
    const int32_t s0 = sidx[n];
    if (s0 < 0) ok = false;
    t.s = s0 < 0 ? 0u : (uint32_t)s0;
    t.hxm = st.hxm;
    t.hxp = st.hxp;
#pragma unroll
    for (int d = 1; d < 7; ++d) {
        uint32_t v = t.s;
        if (PARITY == 1 && st.inx(c7x(d))) {
            const int32_t q = sidx[st.at(c7x(d), c7y(d), c7z(d))];
            if (q < 0) ok = false;
            else v = (uint32_t)q;
        }
        t.nb[d - 1] = v;
    }
    return ok;
}

// AA pattern on the storage: even parity reads slot i of the site and writes
// slot opp(i); odd parity reads slot opp(i) of the upstream neighbour and
// writes slot i of the downstream one (a population leaving through an x face
// stays in the site's own slot).  Population arrays keep the stride N.
template <int PARITY>
__device__ __forceinline__ void gather7(const float* pop, uint32_t N, const SSite& st, float* f) {
    f[0] = pop[st.s];
#pragma unroll
    for (int i = 1; i < 7; ++i) {
        if (PARITY == 0 || !st.inx(-c7x(i))) f[i] = pop[i * N + st.s];
        else f[i] = pop[opp7(i) * N + st.nb[opp7(i) - 1]];
    }
}

template <int PARITY>
__device__ __forceinline__ void scatter7(float* pop, uint32_t N, const SSite& st, const float* f) {
    pop[st.s] = f[0];
#pragma unroll
    for (int i = 1; i < 7; ++i) {
        if (PARITY == 0 || !st.inx(c7x(i))) pop[opp7(i) * N + st.s] = f[i];
        else pop[i * N + st.nb[i - 1]] = f[i];
    }
}

// the same gather for any site, stored or not: a slot whose owner has no
// storage still holds its initial value t_i * c0 (field output only)
template <int PARITY>
__device__ __forceinline__ void gather7_any(const float* pop, uint32_t N, const int32_t* sidx, const Geo& g, int x,
                                            int y, int z, uint32_t n, float c0, float* f) {
    const Site st = make_site(g, x, y, z, n);
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        uint32_t owner = n;
        int idx = i;
        if (PARITY == 1 && i > 0 && st.inx(-c7x(i))) { owner = st.at(-c7x(i), -c7y(i), -c7z(i)); idx = opp7(i); }
        const int32_t so = sidx[owner];
        f[i] = so >= 0 ? pop[idx * N + (uint32_t)so] : t7(idx) * c0;
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
        if (r.ksp > 0.0) {
            double prod = 1.0;
            for (int j = 0; j < r.n_mass; ++j) {
                const double c0 = C[r.mass_s[j] * cs];
                prod *= c0 < THRD ? 0.0 : c0;
            }
            rate *= fmax(prod / r.ksp - 1.0, 0.0);
        } else {
            for (int j = 0; j < r.n_mass; ++j) {
                const double c0 = C[r.mass_s[j] * cs];
                rate *= c0 < THRD ? 0.0 : c0;
            }
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
// ops (the per-operator entry points): bit 1 kinetics, bit 2 surrogate
__device__ __forceinline__ void kinetics_increments(const AdeParams& p, const double* bio, int64_t N, int64_t n,
                                                    const double* Cur, int cs, double* R, double* B, double* BR,
                                                    int bd, int ops = 15) {
    for (int m = 0; m < p.M; ++m) {
        // a microbe solved by LBM: its biomass is its carrier solute's density
        const double b = p.carrier[m] >= 0 ? Cur[p.carrier[m] * cs] : bio[m * N + n];
        B[m * bd] = b < THRD ? 0.0 : b;
    }
    if (p.do_kin && (ops & 1)) {
        rates_dev(p, 0, Cur, cs, B, R, BR, bd);
        for (int s = 0; s < p.S; ++s) {
            const double d = R[s * bd] * p.dt;
            R[s * bd] = (d > THRD || d < -THRD) ? d : 0.0;
        }
        for (int m = 0; m < p.M; ++m) {
            const double d = BR[m * bd] * p.dt;
            BR[m * bd] = (d > THRD || d < -THRD) ? d : 0.0;
        }
        // the dB of a microbe solved by LBM goes to its lattice (update_rxnLattices
        // adds the bFree lattices' dB as it adds the solutes' dC)
        if (p.n_carried)
            for (int m = 0; m < p.M; ++m)
                if (p.carrier[m] >= 0) { R[p.carrier[m] * bd] += BR[m * bd]; BR[m * bd] = 0.0; }
    } else {
        for (int s = 0; s < p.S; ++s) R[s * bd] = 0.0;
        for (int m = 0; m < p.M; ++m) BR[m * bd] = 0.0;
    }
    if (p.n_srg > 0 && (ops & 2)) surrogate_chain(p, Cur, cs, B, R, BR, bd);
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

// run_equilibrium_biotic with the reference's live solver
// (part4_eqsolver.hh:1355-1494 -> calculate_species_concentrations, :1187):
// totals and cold start from the voxel's species, PCF + Anderson, and the
// species it ends at applied through the processor's limiter whether or not
// the solve converged.  Returns 1 if the solve did not converge.
template <int NC>
__device__ __forceinline__ int pcf_voxel(const EqDev& e, int S, int max_iter, double tol, double* Cur, double* App,
                                      int cs, int32_t* iters_out) {
    double T[NC], x[NC];
    pcf_totals_and_start<NC>(e, Cur, cs, T, x);
    int conv = 0;
    const int it = eq_pcf<NC>(e, T, Cur, cs, x, max_iter, tol, e.depth, &conv);
    if (iters_out) *iters_out = it;
    for (int s = 0; s < S && s < e.ns; ++s) {
        const double c0 = Cur[s * cs];
        const double conc = fmax(c0, 1e-30);
        double eqc = e.active[s] ? pcf_species<NC>(e, s, x, conc) : pcf_passive(conc);
        double d = eqc - conc;
        const double mx = fmax(1e-9, 0.1 * fabs(conc));
        if (fabs(d) > mx) d = d > 0 ? mx : -mx;
        if (conc + d < 1e-20) d = 1e-20 - conc;
        if (fabs(d) > THRD) { Cur[s * cs] += d; App[s * cs] += d; }
    }
    return conv ? 0 : 1;
}

// The reaction chain of one voxel.  Cur holds the current densities (updated
// as each processor applies its increments), App the total increment per
// solute.  Returns 1 if the equilibrium solve did not converge.
// ops selects processors for the per-operator entry points (bit 1 kinetics,
// 2 surrogate, 4 abiotic + dissolution, 8 equilibrium); the step runs all.
template <int NC, int SOLVER>
__device__ int reaction_chain(const AdeK& k, int64_t n, uint32_t sto, int x, int y, int z, uint8_t cls, double* Cur,
                              double* App,
                              int cs, double* R, double* B, double* BR, int bd, int ops = 15) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N;
    int nonconv = 0;
    // kinetics and surrogate increments; update_rxnLattices (:338-429) applies
    // the sums that exceed thrd
    if ((p.do_kin && (ops & 1)) || (p.n_srg > 0 && (ops & 2))) {
        kinetics_increments(p, k.bio, N, n, Cur, cs, R, B, BR, bd, ops);
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
    const bool abio = p.do_abio && (ops & 4) && (!p.surface_only || (cls & F_SURFACE));
    const bool dis = p.do_dissol && (ops & 4) && (cls & (F_PHASE_NBR | F_PHASE_SELF));
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
        if (!(ops & 8)) return nonconv;
        const EqDev& e = k.e;
        if constexpr (SOLVER == CL_EQ_SOLVER_PCF) {
            int32_t it = 0;
            nonconv = pcf_voxel<NC>(e, p.S, p.eq.max_iter, p.eq.tol, Cur, App, cs, &it);
            if (k.eq_iters) k.eq_iters[n] = it;
            return nonconv;
        }
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
        double xprev[NC];
        if (k.eq_x) {
            warm = true;
            bool two = true;
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                xprev[j] = (double)k.eq_x[(int64_t)j * N + sto];
                warm = warm && (xprev[j] == xprev[j]);
                const double xq = (double)k.eq_xp[(int64_t)j * N + sto];
                two = two && (xq == xq);
                x[j] = xprev[j];
                if (two) x[j] = fmin(fmax(2.0 * xprev[j] - xq, -30.0), 1.0);
            }
            // the linear extrapolation of the last two solutions, or the last one
            if (!two) {
#pragma unroll
                for (int j = 0; j < NC; ++j) x[j] = xprev[j];
            }
        }
        // the warm attempt (previous solution, warm_iter iterations), then the
        // cold start; one call site keeps one copy of the solver in the kernel
        for (int phase = warm ? 0 : 1; phase < 2; ++phase) {
            if (phase == 1) cold(x);
            it += eq_newton<NC>(e, T, x, phase == 0 ? p.eq.warm_iter : p.eq.max_iter, p.eq.tol, &conv, nullptr, R,
                                bd);
            if (conv) break;
        }
        if (k.eq_x && conv) {
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                k.eq_xp[(int64_t)j * N + sto] = (float)xprev[j];
                k.eq_x[(int64_t)j * N + sto] = (float)x[j];
            }
        }
        if (k.eq_iters) k.eq_iters[n] = it;
        if (!conv) nonconv = 1;
        else {
            for (int s = 0; s < p.S && s < e.ns; ++s) {
                const double conc = fmax(Cur[s * cs], 1e-30);
                // the species of the converged point: kept by the last evaluation
                // (the R column is free during the solve), else recomputed
                double eqc = !e.active[s] ? fmin(conc, 10.0) : (NC <= 3 ? R[s * bd] : species_c<NC>(e, s, x));
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

// ---------------------------------------------------------------------------
// The step as two launches over the interior.
//
// Both run over the live list (the interior sites that stream, in site
// order; rebuilt when the classes change).
//
// ade_react_kernel: one thread per entry, the reactive ones working (all but
// coupled NoDynamics sites).  It gathers the site's populations of this step
// (pre-collision; the BGK collision keeps each density, so they are the
// densities the reference's processors read after collide), runs the reaction
// chain on shared-memory columns of its own, applies the immobile and biomass
// increments, and writes the mobile solutes' total increments to dc.  Its
// warps hold only reactive sites and wait on no barrier, so the FP64 chain
// runs on full warps at the occupancy its registers allow.
//
// ade_stream_kernel: one thread per entry: gather, collide (or the
// bounce-back swap of a reopened grain), add t_i * dc, scatter.  No FP64, no
// shared memory, and no idle lanes: the solid sites a full-lattice traversal
// would mask off are not on the list, so every lane has loads in flight.
//
// Both read the same populations of the step; the second read comes from L2
// for the part still resident and from HBM otherwise.
constexpr int kReactBlock = 128;

template <int NMOB, int NC, int PARITY, int SOLVER>
__global__ void __launch_bounds__(kReactBlock, 4)
ade_react_kernel(const __grid_constant__ AdeK k, const uint32_t* __restrict__ list, int64_t r0, int64_t count,
                 float* __restrict__ dc) {
    extern __shared__ double sm[];
    const int t = threadIdx.x;
    const AdeParams& p = k.p;
    const int Mw = p.M > 0 ? p.M : 1;
    double* Cur = sm;                           // [S][kReactBlock]
    double* App = Cur + p.S * kReactBlock;      // [S][kReactBlock]
    double* Rw = App + p.S * kReactBlock;       // [S][kReactBlock]
    double* Bw = Rw + p.S * kReactBlock;        // [M][kReactBlock]
    double* BRw = Bw + Mw * kReactBlock;        // [M][kReactBlock]
    const int64_t N = k.g.N;
    const uint32_t N32 = (uint32_t)N;
    unsigned long long nonconv = 0;
    double* cCur = Cur + t;
    double* cApp = App + t;
    for (int64_t r = r0 + (int64_t)blockIdx.x * kReactBlock + t; r < count; r += (int64_t)gridDim.x * kReactBlock) {
        const uint32_t n = list[r];
        const uint8_t cls = k.cls[n];
        if (!(cls & F_REACTIVE)) continue;            // streams, does not react (a coupled NoDynamics site)
        int x, y, z;
        decode(k.g, n, x, y, z);
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) atomicAdd(&k.counters[1], 1ull);
        for (int s = 0; s < p.S; ++s) cApp[s * kReactBlock] = 0.0;
#pragma unroll
        for (int m0 = 0; m0 < NMOB; m0 += kGroup) {
            float f[kGroup][7];
#pragma unroll
            for (int g = 0; g < kGroup; ++g)
                if (m0 + g < NMOB) gather7<PARITY>(k.pop + (int64_t)(m0 + g) * 7 * N, N32, st, f[g]);
#pragma unroll
            for (int g = 0; g < kGroup; ++g) {
                if (m0 + g >= NMOB) continue;
                float rr = 0.f;
#pragma unroll
                for (int i = 0; i < 7; ++i) rr += f[g][i];
                cCur[p.mob_index[m0 + g] * kReactBlock] = (double)rr;
            }
        }
        for (int s = 0; s < p.S; ++s)
            if (p.mob_slot[s] < 0) cCur[s * kReactBlock] = k.imm[(int64_t)s * N + n];
        nonconv += reaction_chain<NC, SOLVER>(k, n, st.s, x, y, z, cls, cCur, cApp, kReactBlock, Rw + t, Bw + t, BRw + t,
                                      kReactBlock);
        for (int s = 0; s < p.S; ++s)
            if (p.mob_slot[s] < 0 && cApp[s * kReactBlock] != 0.0) k.imm[(int64_t)s * N + n] += cApp[s * kReactBlock];
#pragma unroll
        for (int m = 0; m < NMOB; ++m) dc[(int64_t)m * N + st.s] = (float)cApp[p.mob_index[m] * kReactBlock];
    }
    for (int o = 16; o > 0; o >>= 1) nonconv += __shfl_down_sync(0xffffffffu, nonconv, o);
    if ((t & 31) == 0 && nonconv) atomicAdd(&k.counters[0], nonconv);
}

template <int NMOB, int PARITY>
__global__ void __launch_bounds__(256, 2) ade_stream_kernel(const __grid_constant__ AdeK k,
                                                          const float* __restrict__ dc, int any_rxn,
                                                          const uint32_t* __restrict__ list, int64_t r0,
                                                          int64_t r1) {
    const AdeParams& p = k.p;
    const int64_t N = k.g.N, plane = k.g.plane;
    const uint32_t N32 = (uint32_t)N;
    // one thread per live site (bounce-back sites are a no-op of the AA step
    // and stay off the list), so every lane of a warp has loads in flight
    for (int64_t r = r0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < r1;
         r += (int64_t)gridDim.x * blockDim.x) {
        const uint32_t n = list[r];
        const uint8_t cls = k.cls[n];
        const uint8_t dyn = cls & 3;
        int x, y, z;
        decode(k.g, n, x, y, z);
        const bool rc = any_rxn && (cls & F_REACTIVE);
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, n, st)) atomicAdd(&k.counters[1], 1ull);
        const float ux = k.u[n], uy = k.u[N + n], uz = k.u[2 * N + n];
        const bool adj = (x == 1 || x == k.g.nx - 2);
        constexpr int kSG = stream_group<PARITY>();
#pragma unroll
        for (int m0 = 0; m0 < NMOB; m0 += kSG) {
            float f[kSG][7];
#pragma unroll
            for (int g = 0; g < kSG; ++g)
                if (m0 + g < NMOB) gather7<PARITY>(k.pop + (int64_t)(m0 + g) * 7 * N, N32, st, f[g]);
#pragma unroll
            for (int g = 0; g < kSG; ++g) {
                const int m = m0 + g;
                if (m >= NMOB) continue;
                float rho = 0.f;
                if (dyn == BB) {
#pragma unroll
                    for (int i = 1; i < 4; ++i) { const float tmp = f[g][i]; f[g][i] = f[g][i + 3]; f[g][i + 3] = tmp; }
                } else if (dyn != NODYN) {
                    const float om = (dyn == BIO) ? p.omega_bio[m] : p.omega_pore[m];
                    collide7(f[g], om, ux, uy, uz, rho);
                } else if (adj) {
#pragma unroll
                    for (int i = 0; i < 7; ++i) rho += f[g][i];
                }
                const float d = rc ? dc[(int64_t)m * N + st.s] : 0.f;
                if (d != 0.f) {
#pragma unroll
                    for (int i = 0; i < 7; ++i) f[g][i] += t7(i) * d;
                }
                if (adj && dyn != BB) {
                    const int side = (x == 1) ? 0 : 1;
                    k.rho_adj[((int64_t)m * 2 + side) * plane + (n - (int64_t)x * plane)] = rho;
                }
            }
#pragma unroll
            for (int g = 0; g < kSG; ++g)
                if (m0 + g < NMOB) scatter7<PARITY>(k.pop + (int64_t)(m0 + g) * 7 * N, N32, st, f[g]);
        }
    }
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
        SSite st;
        if (!make_ssite<PARITY>(k.g, k.sidx, x, y, z, (uint32_t)n, st)) atomicAdd(&k.counters[1], 1ull);
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
    k.eq_xp = c->d_eq_xp;
    k.mask = c->d_mask;
    k.phase = c->d_phase;
    k.rel = c->d_rel;
    k.counters = c->d_counters;
    k.sidx = c->d_sidx;
    k.learn_w = nullptr;
    k.learn_norm = nullptr;
    k.pair_T = k.pair_X = nullptr;
    k.pair_count = nullptr;
    k.pair_cap = 0;
    k.pair_salt = (uint32_t)(c->step_index * 0x632BE5ABu);
    k.pair_mask = (1u << c->learn_shift) - 1u;
    if (c->learn && c->learn_interval > 0) {
        k.pair_T = c->d_pair_T;
        k.pair_X = c->d_pair_X;
        k.pair_count = c->d_pair_count;
        k.pair_cap = c->pair_cap;
        if (c->learn_ready) {
            int trained = 0;
            eq_solver_network(c->learn, &k.learn_w, &k.learn_norm, &trained);
            if (!trained) k.learn_w = k.learn_norm = nullptr;
        }
    }
    k.nodyn_coupled = c->ade_nodyn_coupled ? 1 : 0;
    k.parity = c->ade_parity;
    k.p = c->ap;
    eqdev_from_system(c->cfg.eq, k.e);
    return k;
}

// the phase voxels' releases of this step (dissolution.cu), before the fused launch
int dissol_release(Ctx* c, const AdeK& k);

template <int NMOB, int NC, int PARITY, int SOLVER>
inline int launch_react_as(Ctx* c, const AdeK& k, cudaStream_t st, int64_t r0, int64_t r1, int rblocks,
                           size_t smem) {
    auto kern = ade_react_kernel<NMOB, NC, PARITY, SOLVER>;
    CL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kern<<<rblocks, kReactBlock, smem, st>>>(k, c->d_live, r0, r1, c->d_dc);
    CL_LAUNCH_CHECK("ade_react_kernel");
    c->launches += 1;
    return CL_OK;
}

// the reaction launch over list entries [r0, r1); the PCF solver (equilibrium
// components only) is a separate instantiation so the Newton one keeps its
// registers
template <int NMOB, int NC>
inline int launch_react(Ctx* c, const AdeK& k, cudaStream_t st, int64_t r0, int64_t r1, int max_blocks) {
    const int S = c->ap.S, M = c->ap.M > 0 ? c->ap.M : 1;
    const size_t smem = (size_t)(3 * S + 2 * M) * kReactBlock * sizeof(double);
    const int rblocks = grid_for(r1 - r0, kReactBlock, max_blocks);
    constexpr int PCF = NC > 0 ? CL_EQ_SOLVER_PCF : CL_EQ_SOLVER_NEWTON;
    const bool pcf = NC > 0 && k.e.solver == CL_EQ_SOLVER_PCF;
    if (c->ade_parity == 0)
        return pcf ? launch_react_as<NMOB, NC, 0, PCF>(c, k, st, r0, r1, rblocks, smem)
                   : launch_react_as<NMOB, NC, 0, CL_EQ_SOLVER_NEWTON>(c, k, st, r0, r1, rblocks, smem);
    return pcf ? launch_react_as<NMOB, NC, 1, PCF>(c, k, st, r0, r1, rblocks, smem)
               : launch_react_as<NMOB, NC, 1, CL_EQ_SOLVER_NEWTON>(c, k, st, r0, r1, rblocks, smem);
}

template <int NMOB>
inline int launch_stream(Ctx* c, const AdeK& k, cudaStream_t st, int64_t r0, int64_t r1, int any_rxn, int max_blocks) {
    if (r1 <= r0) return CL_OK;
    const int blocks = grid_for(r1 - r0, 256, max_blocks);
    if (c->ade_parity == 0) ade_stream_kernel<NMOB, 0><<<blocks, 256, 0, st>>>(k, c->d_dc, any_rxn, c->d_live, r0, r1);
    else ade_stream_kernel<NMOB, 1><<<blocks, 256, 0, st>>>(k, c->d_dc, any_rxn, c->d_live, r0, r1);
    CL_LAUNCH_CHECK("ade_stream_kernel");
    c->launches += 1;
    return CL_OK;
}

template <int NMOB, int NC>
inline int launch_step(Ctx* c, const AdeK& k) {
    const bool any_rxn = c->ap.do_kin || c->ap.do_abio || c->ap.n_srg > 0 || c->ap.do_dissol || NC > 0;
    int r = CL_OK;
    if (c->store_dirty && (r = store_update(c, 0))) return r;
    if (c->live_dirty && (r = build_live_list(c))) return r;
    if (any_rxn && c->ap.do_dissol && (r = dissol_release(c, k))) return r;
    const int G = any_rxn ? c->slabs : 1;
    if (G <= 1) {
        if (any_rxn && c->n_live > 0) {
            if ((r = timing_begin(c, CL_KERNEL_ADE_REACT))) return r;
            if ((r = launch_react<NMOB, NC>(c, k, c->stream, 0, c->n_live, 148 * 4 * 8))) return r;
            if ((r = timing_end(c, CL_KERNEL_ADE_REACT))) return r;
        }
        if ((r = timing_begin(c, CL_KERNEL_ADE_MAIN))) return r;
        if ((r = launch_stream<NMOB>(c, k, c->stream, 0, c->n_live, any_rxn ? 1 : 0, 148 * 8))) return r;
        if ((r = timing_end(c, CL_KERNEL_ADE_MAIN))) return r;
    } else {
        // slab j's reactions (s_react) then its streaming (s_stream, after the
        // reactions of slab j); slab j+1's reactions overlap slab j's streaming.
        // The two touch disjoint population slots: a site's AA read and write
        // sets coincide, so slabs of sites never share a slot.
        // grids of four blocks per SM each, so that both launches fit on an SM
        const int rmax = 148 * 4, smax = 148 * 4;
        if ((r = timing_begin(c, CL_KERNEL_ADE_MAIN))) return r;
        CL_CUDA(cudaEventRecord(c->ev_fork, c->stream));
        CL_CUDA(cudaStreamWaitEvent(c->s_react, c->ev_fork, 0));
        CL_CUDA(cudaStreamWaitEvent(c->s_stream, c->ev_fork, 0));
        for (int j = 0; j < G; ++j) {
            const int64_t r0 = c->slab_live[j], r1 = c->slab_live[j + 1];
            if (r1 > r0 && (r = launch_react<NMOB, NC>(c, k, c->s_react, r0, r1, rmax))) return r;
            CL_CUDA(cudaEventRecord(c->ev_slab[j], c->s_react));
            CL_CUDA(cudaStreamWaitEvent(c->s_stream, c->ev_slab[j], 0));
            if ((r = launch_stream<NMOB>(c, k, c->s_stream, r0, r1, 1, smax))) return r;
        }
        CL_CUDA(cudaEventRecord(c->ev_join, c->s_stream));
        CL_CUDA(cudaStreamWaitEvent(c->stream, c->ev_join, 0));
        if ((r = timing_end(c, CL_KERNEL_ADE_MAIN))) return r;
    }
    c->launches += 1;
    const int bblocks = grid_for(2 * c->geo.plane, 256, 148 * 4);
    if (c->ade_parity == 0) ade_boundary_kernel<NMOB, 0><<<bblocks, 256, 0, c->stream>>>(k);
    else ade_boundary_kernel<NMOB, 1><<<bblocks, 256, 0, c->stream>>>(k);
    CL_LAUNCH_CHECK("ade_boundary_kernel");
    c->ade_parity ^= 1;
    return CL_OK;
}

// one translation unit per component count instantiates these
int ade_step_nc0(Ctx* c); int ade_step_nc1(Ctx* c); int ade_step_nc2(Ctx* c);
int ade_step_nc3(Ctx* c); int ade_step_nc4(Ctx* c); int ade_step_nc5(Ctx* c);

}  // namespace cl
