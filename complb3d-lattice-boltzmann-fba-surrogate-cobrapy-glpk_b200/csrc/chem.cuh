// chem.cuh -- chemistries compiled into the library.
//
// The reference compiles its rate laws into the program: the user edits
// defineKinetics.hh / defineAbioticKinetics.hh and rebuilds, and
// run_kinetics calls defineRxnKinetics once per voxel with the voxel's
// concentrations and biomass (src/complab3d_processors_part1.hh:63-146,
// defineKinetics.hh:223).  This header is that hook on the device: a
// chemistry is a type that fixes, at compile time, how many solutes and
// microbes there are, which solutes are mobile, how many equilibrium
// components the tableau has, and the structure of its rate laws.  The
// values (rate constants, half-saturations, logK, relaxation, boundary
// values) stay run-time inputs in cl_config; a chemistry may also fix its
// tableau's stoichiometry (Tab = TabFixed<...>), which the configuration must
// then hold exactly, so that its Newton solve folds every zero coefficient.
//
// With every size known, the transport step keeps a voxel's whole state in
// registers and unrolls every loop over solutes, species and reactions (the
// fused launch of ade_fast.cuh); configurations that match no compiled
// chemistry run the run-time-table launches of ade_kernels.cuh.
//
// A chemistry provides
//   S, NMOB, M, NC                  solutes, mobile solutes, microbes, components
//   mobile(s), slot(s)              whether solute s has a lattice, and its slot
//   matches(cfg)                    host: the configuration has this structure
//   kinetics(p, C, B, R, BR, mask)  rates per second (defineRxnKinetics); B floored
//                                   at thrd, C as stored
//   abiotic(p, C, R, mask)          rates per second (defineAbioticRxnKinetics)
//   Tab                             the tableau the Newton solve reads: TabRun
//                                   (cl_config's) or TabFixed (compiled in)
//   kSrg, Consts                    whether the step runs surrogate networks
//                                   (surrogate(p, consts, C, B, D, DB)), and the
//                                   constants the kernel takes for them
// Rates follow the run-time table's arithmetic (rates_dev) term for term, so
// a configuration runs to the same numbers on either launch.
#pragma once
#include <cmath>
#include "internal.h"
#include "newton.cuh"
#include "../../include/complab_ratelaw.hpp"

namespace cl {

#ifndef THRD
#define THRD 1e-12
#endif

// ---- building blocks of table-shaped rate laws --------------------------------
// C/(Ks+C) with C below thrd read as zero (run_kinetics floors C first)
__host__ __device__ __forceinline__ double chem_monod(double c0, double ks) {
    const double c = c0 < THRD ? 0.0 : c0;
    return c / (ks + c);
}
__host__ __device__ __forceinline__ double chem_mass(double c0) { return c0 < THRD ? 0.0 : c0; }

// subsR[s] += nu[s] * rate for every solute (the table's stoichiometry row)
template <int S>
__host__ __device__ __forceinline__ void chem_add(const cl_rxn& r, double rate, double (&R)[S]) {
#pragma unroll
    for (int s = 0; s < S; ++s) R[s] = fma(r.nu[s], rate, R[s]);
}

// the table's closing steps: decay of every microbe, then non-finite rates zeroed
template <int S, int MW>
__host__ __device__ __forceinline__ void chem_close_biotic(const AdeParams& p, int M, const double (&B)[MW],
                                                           double (&R)[S], double (&BR)[MW]) {
#pragma unroll
    for (int m = 0; m < MW; ++m)
        if (m < M) BR[m] -= p.decay[m] * fmax(B[m], 0.0);
#pragma unroll
    for (int s = 0; s < S; ++s) if (!isfinite(R[s])) R[s] = 0.0;
#pragma unroll
    for (int m = 0; m < MW; ++m) if (m < M && !isfinite(BR[m])) BR[m] = 0.0;
}
template <int S>
__host__ __device__ __forceinline__ void chem_close_abiotic(double (&R)[S]) {
#pragma unroll
    for (int s = 0; s < S; ++s) if (!isfinite(R[s])) R[s] = 0.0;
}

// host-side structure checks of a table entry
inline bool rxn_is(const cl_rxn& r, int microbe, std::initializer_list<int> monod, std::initializer_list<int> mass) {
    if (r.microbe != microbe || r.n_monod != (int)monod.size() || r.n_mass != (int)mass.size()) return false;
    int j = 0;
    for (int s : monod) if (r.monod_s[j++] != s) return false;
    j = 0;
    for (int s : mass) if (r.mass_s[j++] != s) return false;
    return true;
}

// ---- the coupled flow + 8-solute chemistry --------------------------------------
// Solutes 0..7 mobile (DOC, O2, NO3-, HCO3-, Ca2+, H+, CO3--, CaCO3(aq)), 8 an
// immobile mineral (CaCO3(s)); one sessile microbe.
//   reaction 0  microbe 0: k B  DOC/(Ks+DOC)  O2/(Ks+O2)      (aerobic oxidation)
//   reaction 1  microbe 0: k B  DOC/(Ks+DOC)  NO3/(Ks+NO3)    (denitrification)
//   reaction 2  abiotic:   k [Ca2+][CO3--], or k (Omega - 1)+ with a Ksp (precipitation)
// Equilibrium: 3 components, CO3-- (species 6), Ca2+ (4) and H+ (5), with
// HCO3- (3) = CO3-- + H+ and CaCO3(aq) (7) = CO3-- + Ca2+ (stoichiometry
// compiled in, logK from the run).
// what a chemistry passes to the fused kernel besides AdeK (in the kernel's
// parameter space): nothing, for a chemistry without networks
struct NoConsts { int unused; };

struct ChemCoupled {
    static constexpr int kId = 1;
    static constexpr const char* kName = "coupled carbonate (8 mobile + 1 mineral, dual Monod, 3 components)";
    static constexpr int S = 9, NMOB = 8, M = 1, NC = 3, MW = 1;
    static constexpr bool kSrg = false;     // no surrogate networks
    using Consts = NoConsts;
    __host__ __device__ static constexpr bool mobile(int s) { return s < 8; }
    __host__ __device__ static constexpr int slot(int s) { return s; }
    struct Fix {
        static constexpr int ns = S, nc = NC;
        __host__ __device__ static constexpr int coef(int i, int j) {
            return i == 6 ? (j == 0) : i == 4 ? (j == 1) : i == 5 ? (j == 2)
                 : i == 3 ? (j == 0 || j == 2) : i == 7 ? (j == 0 || j == 1) : 0;
        }
        __host__ __device__ static constexpr int comp_species(int j) { return j == 0 ? 6 : j == 1 ? 4 : 5; }
    };
    using Tab = TabFixed<Fix>;
    static bool matches(const cl_config& c) {
        if (c.n_solutes != S || c.n_microbes != M || c.n_rxn != 3 || c.n_srg != 0) return false;
        for (int s = 0; s < S; ++s) if ((c.immobile[s] != 0) == mobile(s)) return false;
        if (!c.use_equilibrium || c.eq.n_comp != NC || c.eq.n_species != S || c.eq.solver != CL_EQ_SOLVER_NEWTON)
            return false;
        for (int i = 0; i < S; ++i)
            for (int j = 0; j < NC; ++j) if (c.eq.stoich[i][j] != (double)Fix::coef(i, j)) return false;
        for (int j = 0; j < NC; ++j) if (c.eq.comp_species[j] != Fix::comp_species(j)) return false;
        return c.rate_law == CL_RATELAW_TABLE && rxn_is(c.rxn[0], 0, {0, 1}, {}) && rxn_is(c.rxn[1], 0, {0, 2}, {}) &&
               rxn_is(c.rxn[2], -1, {}, {4, 6});
    }
    __host__ __device__ static void kinetics(const AdeParams& p, const double (&C)[S], const double (&B)[MW],
                                             double (&R)[S], double (&BR)[MW], int) {
#pragma unroll
        for (int s = 0; s < S; ++s) R[s] = 0.0;
        BR[0] = 0.0;
        const double b = B[0];
        if (b > 0.0) {
            {
                const cl_rxn& r = p.rxn[0];
                double rate = r.k * b;
                rate *= chem_monod(C[0], r.monod_ks[0]);
                rate *= chem_monod(C[1], r.monod_ks[1]);
                chem_add<S>(r, rate, R);
                BR[0] = fma(r.yield, rate, BR[0]);
            }
            {
                const cl_rxn& r = p.rxn[1];
                double rate = r.k * b;
                rate *= chem_monod(C[0], r.monod_ks[0]);
                rate *= chem_monod(C[2], r.monod_ks[1]);
                chem_add<S>(r, rate, R);
                BR[0] = fma(r.yield, rate, BR[0]);
            }
        }
        chem_close_biotic<S, MW>(p, M, B, R, BR);
    }
    __host__ __device__ static void abiotic(const AdeParams& p, const double (&C)[S], double (&R)[S], int) {
#pragma unroll
        for (int s = 0; s < S; ++s) R[s] = 0.0;
        const cl_rxn& r = p.rxn[2];
        double rate = r.k;
        if (r.ksp > 0.0) {
            double prod = 1.0;
            prod *= chem_mass(C[4]);
            prod *= chem_mass(C[6]);
            rate *= fmax(prod / r.ksp - 1.0, 0.0);
        } else {
            rate *= chem_mass(C[4]);
            rate *= chem_mass(C[6]);
        }
        chem_add<S>(r, rate, R);
        chem_close_abiotic<S>(R);
    }
};

// ---- the biotic chemistry of the cellular-automaton workload ----------------------
// Four mobile solutes (electron donor, O2, NO3-, product) and one sessile
// microbe; dual Monod on (donor, O2) and (donor, NO3-); no equilibrium.
struct ChemBiotic4 {
    static constexpr int kId = 2;
    static constexpr const char* kName = "biotic dual Monod (4 mobile solutes, 1 microbe)";
    static constexpr int S = 4, NMOB = 4, M = 1, NC = 0, MW = 1;
    static constexpr bool kSrg = false;     // no surrogate networks
    using Consts = NoConsts;
    using Tab = TabRun;
    __host__ __device__ static constexpr bool mobile(int) { return true; }
    __host__ __device__ static constexpr int slot(int s) { return s; }
    static bool matches(const cl_config& c) {
        if (c.n_solutes != S || c.n_microbes != M || c.n_rxn != 2 || c.n_srg != 0 || c.use_equilibrium) return false;
        for (int s = 0; s < S; ++s) if (c.immobile[s]) return false;
        return c.rate_law == CL_RATELAW_TABLE && rxn_is(c.rxn[0], 0, {0, 1}, {}) && rxn_is(c.rxn[1], 0, {0, 2}, {});
    }
    __host__ __device__ static void kinetics(const AdeParams& p, const double (&C)[S], const double (&B)[MW],
                                             double (&R)[S], double (&BR)[MW], int) {
#pragma unroll
        for (int s = 0; s < S; ++s) R[s] = 0.0;
        BR[0] = 0.0;
        const double b = B[0];
        if (b > 0.0) {
            {
                const cl_rxn& r = p.rxn[0];
                double rate = r.k * b;
                rate *= chem_monod(C[0], r.monod_ks[0]);
                rate *= chem_monod(C[1], r.monod_ks[1]);
                chem_add<S>(r, rate, R);
                BR[0] = fma(r.yield, rate, BR[0]);
            }
            {
                const cl_rxn& r = p.rxn[1];
                double rate = r.k * b;
                rate *= chem_monod(C[0], r.monod_ks[0]);
                rate *= chem_monod(C[2], r.monod_ks[1]);
                chem_add<S>(r, rate, R);
                BR[0] = fma(r.yield, rate, BR[0]);
            }
        }
        chem_close_biotic<S, MW>(p, M, B, R, BR);
    }
    __host__ __device__ static void abiotic(const AdeParams&, const double (&)[S], double (&R)[S], int) {
#pragma unroll
        for (int s = 0; s < S; ++s) R[s] = 0.0;
    }
};

// ---- the reference's default network: the Zhao uranium / iron / sulfur model ----
// The 24-substrate layout (speciation off) with its 12 biomass pools held as
// sessile fields; the rate laws are clrl::zhao (include/complab_ratelaw.hpp),
// called with the concentrations and biomass floored at thrd and the voxel's
// mask, as run_kinetics / run_abiotic_kinetics call defineRxnKinetics /
// defineAbioticRxnKinetics (complab3d_processors_part1.hh:63-249).
struct ChemZhao24 {
    static constexpr int kId = 3;
    static constexpr const char* kName = "Zhao uranium network (24 substrates, 12 biomass pools)";
    static constexpr int S = 24, NMOB = 15, M = 12, NC = 0, MW = 12;
    static constexpr bool kSrg = false;     // no surrogate networks
    using Consts = NoConsts;
    using Tab = TabRun;
    __host__ __device__ static constexpr bool mobile(int s) {
        return !(s == 2 || s == 4 || s == 5 || s == 6 || s == 9 || s == 13 || s == 21 || s == 22 || s == 23);
    }
    // rank of solute s among the mobile ones
    __host__ __device__ static constexpr int slot(int s) {
        int k = 0;
        for (int q = 0; q < s; ++q) k += mobile(q) ? 1 : 0;
        return k;
    }
    static bool matches(const cl_config& c) {
        if (c.rate_law != CL_RATELAW_ZHAO || c.n_solutes != S || c.n_microbes != M || c.n_srg != 0) return false;
        if (c.use_equilibrium || c.dissol_enabled) return false;
        for (int s = 0; s < S; ++s) if ((c.immobile[s] != 0) == mobile(s)) return false;
        return true;
    }
    __host__ __device__ static void kinetics(const AdeParams&, const double (&C)[S], const double (&B)[MW],
                                             double (&R)[S], double (&BR)[MW], int mask) {
        double Cf[S];
#pragma unroll
        for (int s = 0; s < S; ++s) Cf[s] = C[s] < THRD ? 0.0 : C[s];
        clrl::zhao::kinetics(clrl::cspan{B, MW}, clrl::cspan{Cf, S}, clrl::dspan{R, S}, clrl::dspan{BR, MW}, mask);
    }
    __host__ __device__ static void abiotic(const AdeParams&, const double (&C)[S], double (&R)[S], int mask) {
        double Cf[S];
#pragma unroll
        for (int s = 0; s < S; ++s) Cf[s] = C[s] < THRD ? 0.0 : C[s];
        clrl::zhao::abiotic(clrl::cspan{Cf, S}, clrl::dspan{R, S}, mask);
    }
};

// ---- the surrogate workload: two organisms' networks in the step ------------------
// Six mobile solutes and two sessile microbes, no rate table reactions (the
// table's decay of each microbe still applies), the surrogate reaction type
// of two organisms (organism o on microbe o with network o), each network
// 3 -> 20 tanh -> 20 tanh -> 4.  surrogate() is run_surrogate3D
// (src/complab3d_processors_surrogate.hh:94-295) as surrogate_chain of
// ade_kernels.cuh evaluates it, operation for operation, with the network's
// shape compiled in and its weights in the kernel's parameter space, so that
// every weight is an operand of its FMA rather than a load.
struct ChemSurrogate2 {
    static constexpr int kId = 4;
    static constexpr const char* kName = "surrogate rates (6 mobile solutes, 2 organisms, 3-20-20-4 networks)";
    static constexpr int S = 6, NMOB = 6, M = 2, NC = 0, MW = 2;
    static constexpr bool kSrg = true;
    static constexpr int kL = 3;
    __host__ __device__ static constexpr int width(int l) { return l == 0 ? 3 : l == 3 ? 4 : 20; }
    __host__ __device__ static constexpr int poff(int l) {
        int o = 0;
        for (int j = 0; j < l; ++j) o += width(j + 1) * width(j) + width(j + 1);
        return o;
    }
    static constexpr int kP = (20 * 3 + 20) + (20 * 20 + 20) + (4 * 20 + 4);   // parameters per network
    struct Consts { float w[2][kP]; };
    using Tab = TabRun;
    __host__ __device__ static constexpr bool mobile(int) { return true; }
    __host__ __device__ static constexpr int slot(int s) { return s; }
    static bool matches(const cl_config& c) {
        if (c.n_solutes != S || c.n_microbes != M || c.n_rxn != 0 || c.n_srg != 2 || c.use_equilibrium) return false;
        for (int s = 0; s < S; ++s) if (c.immobile[s]) return false;
        for (int o = 0; o < 2; ++o) if (c.srg[o].microbe != o || c.srg[o].net != o) return false;
        return c.rate_law == CL_RATELAW_TABLE;
    }
    // host: the networks set on the context have the compiled shape
    static bool ready(const AdeParams& ap) {
        for (int o = 0; o < 2; ++o) {
            const SrgNetDev& d = ap.net[o];
            if (d.L != kL || !d.params) return false;
            for (int l = 0; l <= kL; ++l) if (d.w[l] != width(l)) return false;
            for (int l = 0; l < kL; ++l) if (d.poff[l] != poff(l)) return false;
        }
        return true;
    }
    // rates_dev with no reactions: the microbes' decay
    __host__ __device__ static void kinetics(const AdeParams& p, const double (&)[S], const double (&B)[MW],
                                             double (&R)[S], double (&BR)[MW], int) {
#pragma unroll
        for (int s = 0; s < S; ++s) R[s] = 0.0;
#pragma unroll
        for (int m = 0; m < MW; ++m) BR[m] = 0.0;
#pragma unroll
        for (int m = 0; m < M; ++m) BR[m] -= p.decay[m] * fmax(B[m], 0.0);
#pragma unroll
        for (int m = 0; m < MW; ++m) if (!isfinite(BR[m])) BR[m] = 0.0;
    }
    __host__ __device__ static void abiotic(const AdeParams&, const double (&)[S], double (&R)[S], int) {
#pragma unroll
        for (int s = 0; s < S; ++s) R[s] = 0.0;
    }
    // the surrogate increments of one voxel, added into D and DB
    __device__ static void surrogate(const AdeParams& p, const Consts& kc, const double (&Cur)[S],
                                     const double (&B)[MW], double (&D)[S], double (&DB)[MW]) {
        bool any = false;
#pragma unroll
        for (int o = 0; o < 2; ++o) any = any || B[o] > THRD;
        if (!any) return;
        double conc[S], draw[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const double c = Cur[s];
            conc[s] = c > THRD ? c : 0.0;
            draw[s] = 0.0;
        }
#pragma unroll
        for (int o = 0; o < 2; ++o) {
            const cl_srg_organism& org = p.srg[o];
            const SrgNetDev& net = p.net[o];
            const double b = B[o];
            if (!(b > THRD)) continue;
            double fin[S];
            const double denom = b * org.mw * p.dt;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const double av = conc[s];
                const double mm = (org.kc[s] + av > 0.0) ? av / (org.kc[s] + av) : 0.0;
                double exh = 0.0;
                if (denom > 1e-30) { exh = -av * 3.6e6 / denom; if (exh < -1e4) exh = -1e4; }
                double v = org.vmax[s] > THRD ? org.vmax[s] * mm : -exh * mm;
                const double cap = -exh;
                if (cap > 0.0 && v > cap) v = cap;
                fin[s] = v;
            }
            float a[20], t[20];
#pragma unroll
            for (int i = 0; i < width(0); ++i) {
                const int kind = org.in_kind[i], idx = org.in_index[i];
                double sel_f = 0.0, sel_c = 0.0;
#pragma unroll
                for (int s = 0; s < S; ++s) if (s == idx) { sel_f = fin[s]; sel_c = conc[s]; }
                float v = kind == CL_SRG_IN_FIN ? (float)sel_f : kind == CL_SRG_IN_CONC ? (float)sel_c : (float)b;
                v = fminf(fmaxf(v, net.xlo[i]), net.xhi[i]);
                a[i] = (v - net.xo[i]) * net.xg[i] + net.xymin;
            }
#pragma unroll
            for (int l = 0; l < kL; ++l) {
                const int wi = width(l), wo = width(l + 1);
                const float* W = kc.w[o] + poff(l);
                // outputs four at a time: unrolled whole, the two networks'
                // code (every weight an immediate operand) overran the
                // instruction cache (3.16 -> 2.68 ms at 256^3 this way)
#pragma unroll 4
                for (int q = 0; q < wo; ++q) {
                    float acc = W[wo * wi + q];
#pragma unroll
                    for (int i = 0; i < wi; ++i) acc = fmaf(W[q * wi + i], a[i], acc);
                    t[q] = (l < kL - 1) ? tanhf(acc) : acc;
                }
#pragma unroll
                for (int q = 0; q < wo; ++q) a[q] = t[q];
            }
            double mu = 0.0;
            double fout[S];
#pragma unroll
            for (int s = 0; s < S; ++s) fout[s] = fin[s];
#pragma unroll
            for (int q = 0; q < width(kL); ++q) {
                const double y = ((double)a[q] - net.yymin) / net.yg[q] + net.yo[q];
                if (org.out_kind[q] == CL_SRG_OUT_GROWTH) mu = y;
                else {
                    const int idx = org.out_index[q];
#pragma unroll
                    for (int s = 0; s < S; ++s) if (s == idx) fout[s] = y;
                }
            }
            if (mu < 1e-8 || !isfinite(mu)) mu = 0.0;
            double dB = (fabs(mu) < THRD) ? -org.kd * b * p.dt : mu * b * p.dt / 3600.0;
            if (dB + b < 0.0) dB = -b;
            if (fabs(dB) > THRD) DB[o] += dB;
#pragma unroll
            for (int s = 0; s < S; ++s) draw[s] += -fout[s] * b * org.mw * p.dt / 3.6e6;
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double d = draw[s];
            if (fabs(d) <= THRD) continue;
            if (d + conc[s] < 0.0) d = -conc[s];
            if (d > 0.0) d = 0.0;
            if (fabs(d) > THRD) D[s] += d;
        }
    }
};

static_assert(ChemSurrogate2::poff(ChemSurrogate2::kL) == ChemSurrogate2::kP, "network size");

}  // namespace cl
