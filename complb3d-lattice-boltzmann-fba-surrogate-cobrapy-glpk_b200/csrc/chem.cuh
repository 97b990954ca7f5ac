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
struct ChemCoupled {
    static constexpr int kId = 1;
    static constexpr const char* kName = "coupled carbonate (8 mobile + 1 mineral, dual Monod, 3 components)";
    static constexpr int S = 9, NMOB = 8, M = 1, NC = 3, MW = 1;
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

}  // namespace cl
