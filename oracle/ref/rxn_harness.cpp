/*
 * rxn_harness.cpp -- the reference's own reaction processors, compiled from
 * the reference tree (oracle/Makefile) and run on one block, to pin the
 * oracle's reaction stage (oracle.c, orc_reaction_stage) and its node
 * conversions.  Test infrastructure only.
 *
 *   ref_rxn_stage   the reaction stage of src/complab.cpp:1264-1374 on the
 *                   current densities: dC = dC0, run_kinetics (part1.hh:63-146)
 *                   -> update_rxnLattices (:338-429) -> dC = dC0 ->
 *                   surfaceAbioticKinetics3D (precipitationVOP.hh:53-145) or
 *                   run_abiotic_kinetics (part1.hh:158-249) ->
 *                   surfaceDissolutionKinetics3D (dissolutionVOP.hh:265-435) ->
 *                   update_abiotic_rxnLattices (part1.hh:258-336) ->
 *                   run_equilibrium_biotic (part4_eqsolver.hh:1322-1494, with
 *                   the reference's PCF + Anderson EquilibriumChemistry).
 *   ref_precip_convert   precipNodeConversion3D (precipitationVOP.hh:158-219).
 *   ref_dissol_convert   dissolNodeConversion3D (dissolutionVOP.hh:459-527).
 *
 * The rate laws are the example headers' own: defineRxnKinetics of
 * examples/05_biotic_cellular_automaton (Monod growth, two microbes),
 * defineAbioticRxnKinetics of examples/13_precipitation (Fe + HS -> FeS) and
 * defineDissolutionRate of examples/14_dissolution (calcite, k H mineral).
 * They are included inside an unnamed namespace before the processor headers
 * (whose own includes of the top-level rate headers their guards then skip),
 * so they bind to the processors here and clash with nothing else in the
 * library.
 */
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <random>
#include <string>
#include <vector>
#include "plb_ca_stub.h"

namespace plb {
template<typename T1, template<typename U> class D1, typename T2, template<typename U> class D2>
class BoxProcessingFunctional3D_LL { public: virtual ~BoxProcessingFunctional3D_LL() {} };
template<typename T1, template<typename U> class D1, typename T2>
class BoxProcessingFunctional3D_LS { public: virtual ~BoxProcessingFunctional3D_LS() {} };
template<typename T1, template<typename U> class D1> class BounceBack { public: BounceBack() {} };
template<typename T1, template<typename U> class D1> class IncBGKdynamics { public: explicit IncBGKdynamics(T1) {} };
template<typename T1> class ScalarField3D;
}
#define COMPLAB_THRD 1e-14            /* src/complab_functions.hh:64 */
#define g_updRxn_debug g_updRxn_debug_rxn_harness   /* part1.hh:54 defines it; the CA harness does too */

namespace {
#include "examples/05_biotic_cellular_automaton/defineKinetics.hh"
}
#if defined(RXN_HARNESS_DISSOLUTION)
namespace {
#include "examples/14_dissolution/defineAbioticKinetics.hh"
}
#else
namespace {
#include "examples/13_precipitation/defineAbioticKinetics.hh"
}
#endif

#include "src/complab3d_processors_part1.hh"
#include "src/precipitationVOP.hh"
#include "src/dissolutionVOP.hh"
#include "src/complab3d_processors_part4_eqsolver.hh"

typedef plb::BlockLattice3D<double, CaStubD3Q7> Lat;

namespace {

struct Grid {
    plint nx, ny, nz;
    std::vector<Lat*> lats;
    Grid(plint nx_, plint ny_, plint nz_, size_t count) : nx(nx_), ny(ny_), nz(nz_) {
        for (size_t i = 0; i < count; ++i) lats.push_back(new Lat(nx, ny, nz));
    }
    ~Grid() { for (auto* p : lats) delete p; }
    size_t idx(plint x, plint y, plint z) const { return ((size_t)x * ny + (size_t)y) * nz + (size_t)z; }
    template<class F> void each(F f) const {
        for (plint x = 0; x < nx; ++x) for (plint y = 0; y < ny; ++y) for (plint z = 0; z < nz; ++z) f(x, y, z, idx(x, y, z));
    }
    void put(Lat* l, const double* v) { each([&](plint x, plint y, plint z, size_t n) { l->setScalar(x, y, z, v[n]); }); }
    void put8(Lat* l, const uint8_t* v) { each([&](plint x, plint y, plint z, size_t n) { l->setScalar(x, y, z, v[n]); }); }
    void zero(Lat* l) { each([&](plint x, plint y, plint z, size_t) { l->setScalar(x, y, z, 0.0); }); }
    void get(Lat* l, double* v) { each([&](plint x, plint y, plint z, size_t n) { v[n] = l->get(x, y, z).computeDensity(); }); }
    void get8(Lat* l, uint8_t* v) {
        each([&](plint x, plint y, plint z, size_t n) { v[n] = (uint8_t)util::roundToInt(l->get(x, y, z).computeDensity()); });
    }
    Box3D box() const { return Box3D{0, nx - 1, 0, ny - 1, 0, nz - 1}; }
};

DissolutionConfig dissol_config(int n_phases, const int* ids, const int* materials, const int* substrates,
                                const double* full, const int* is_precip, double reopen, int surface_only) {
    DissolutionConfig d;
    d.enabled = n_phases > 0;
    d.reopen_fraction = reopen;
    d.surface_only = surface_only;
    for (int k = 0; k < n_phases; ++k) {
        SolidPhase p;
        p.id = ids[k]; p.material_number = materials[k]; p.substrate = substrates[k];
        p.full_density = full[k]; p.initial_fill = full[k]; p.is_precipitate = is_precip[k] != 0;
        d.phases.push_back(p);
    }
    return d;
}

}  // namespace

extern "C" {

/* flags: 1 kinetics, 2 abiotic, 4 abiotic surface gate, 8 dissolution,
 * 16 equilibrium.  C: S*N densities in/out; B: M*N in/out; phase: N ids.
 * The equilibrium tableau: stoich ns x nc (ns = S), logk ns, comp_species nc. */
int ref_rxn_stage(int nx, int ny, int nz, int S, int M, double dt, int solid, int bb, int flags,
                  const uint8_t* mask, const uint8_t* phase, double* C, double* B,
                  int n_phases, const int* ids, const int* materials, const int* substrates, const double* full,
                  const int* is_precip, double reopen, int surface_only, const int* pore, int n_pore,
                  int nc, const double* stoich, const double* logk, const int* comp_species,
                  int eq_max_iter, double eq_tol, int eq_depth) {
    const size_t N = (size_t)nx * ny * nz;
    // [C.., B.., dC.., dB.., mask, phase]
    Grid g(nx, ny, nz, (size_t)2 * (S + M) + 2);
    std::vector<Lat*>& L = g.lats;
    for (int s = 0; s < S; ++s) g.put(L[s], C + s * N);
    for (int m = 0; m < M; ++m) g.put(L[S + m], B + m * N);
    Lat* maskL = L[2 * (S + M)];
    Lat* phaseL = L[2 * (S + M) + 1];
    g.put8(maskL, mask);
    g.put8(phaseL, phase);
    auto dC = [&](int s) { return L[S + M + s]; };
    auto dB = [&](int m) { return L[2 * S + M + m]; };
    auto reset = [&]() { for (int s = 0; s < S; ++s) g.zero(dC(s)); for (int m = 0; m < M; ++m) g.zero(dB(m)); };
    std::vector<Lat*> kns;                      // ptr_kns_lattices (complab.cpp:901-913)
    for (int s = 0; s < S; ++s) kns.push_back(L[s]);
    for (int m = 0; m < M; ++m) kns.push_back(L[S + m]);
    for (int s = 0; s < S; ++s) kns.push_back(dC(s));
    for (int m = 0; m < M; ++m) kns.push_back(dB(m));
    kns.push_back(maskL);
    std::vector<Lat*> abio;                     // ptr_abiotic_kns_lattices (:1008-1010)
    for (int s = 0; s < S; ++s) abio.push_back(L[s]);
    for (int s = 0; s < S; ++s) abio.push_back(dC(s));
    abio.push_back(maskL);
    std::vector<Lat*> dis(abio);                // ptr_dissol (:878-881)
    dis.push_back(phaseL);
    std::vector<Lat*> eq;                       // ptr_eq_lattices (:1060-1061)
    for (int s = 0; s < S; ++s) eq.push_back(L[s]);
    eq.push_back(maskL);
    std::vector<plint> pores(pore, pore + n_pore);
    DissolutionConfig dcfg = dissol_config(n_phases, ids, materials, substrates, full, is_precip, reopen, surface_only);

    reset();                                    // dC = dC0; dBp = dBp0; dBf = dBf0 (:1264)
    if (flags & 1) {
        std::vector<std::vector<double>> kc;
        std::vector<double> mu;
        run_kinetics<double, CaStubD3Q7> k(nx, S, M, dt, kc, mu, solid, bb);
        k.process(g.box(), kns);
        update_rxnLattices<double, CaStubD3Q7> u(nx, S, M, solid, bb);
        u.process(g.box(), kns);
    }
    if (flags & 2) {
        reset();                                // dC = dC0 (:1328)
        if (flags & 4) {
            surfaceAbioticKinetics3D<double, CaStubD3Q7> a(nx, ny, nz, S, dt, solid, bb, 1);
            a.process(g.box(), abio);
        } else {
            run_abiotic_kinetics<double, CaStubD3Q7> a(nx, S, dt, solid, bb);
            a.process(g.box(), abio);
        }
        if (flags & 8) {
            surfaceDissolutionKinetics3D<double, CaStubD3Q7> d(nx, ny, nz, S, dt, solid, bb, pores, &dcfg);
            d.process(g.box(), dis);
        }
        update_abiotic_rxnLattices<double, CaStubD3Q7> u(nx, S, solid, bb);
        u.process(g.box(), abio);
    } else if (flags & 8) {
        reset();                                // :1359-1366
        surfaceDissolutionKinetics3D<double, CaStubD3Q7> d(nx, ny, nz, S, dt, solid, bb, pores, &dcfg);
        d.process(g.box(), dis);
        update_abiotic_rxnLattices<double, CaStubD3Q7> u(nx, S, solid, bb);
        u.process(g.box(), abio);
    }
    if (flags & 16) {
        EquilibriumChemistry<double> chem;
        std::vector<std::string> sn(S), cn(nc);
        for (int i = 0; i < S; ++i) sn[i] = "S" + std::to_string(i);
        for (int j = 0; j < nc; ++j) cn[j] = comp_species[j] >= 0 ? sn[comp_species[j]] : "C" + std::to_string(j);
        chem.setSpeciesNames(sn);
        chem.setComponentNames(cn);
        chem.setLogK(std::vector<double>(logk, logk + S));
        std::vector<std::vector<double>> st(S, std::vector<double>(nc));
        for (int i = 0; i < S; ++i) for (int j = 0; j < nc; ++j) st[i][j] = stoich[i * nc + j];
        chem.setStoichiometryMatrix(st);
        chem.setMaxIterations(eq_max_iter);
        chem.setTolerance(eq_tol);
        chem.setAndersonDepth(eq_depth);
        run_equilibrium_biotic<double, CaStubD3Q7> e(nx, S, chem, solid, bb);
        e.process(g.box(), eq);
    }
    for (int s = 0; s < S; ++s) g.get(L[s], C + s * N);
    for (int m = 0; m < M; ++m) g.get(L[S + m], B + m * N);
    return 0;
}

/* precipNodeConversion3D on [P, mask, phase]; returns voxels whose mask changed */
long long ref_precip_convert(int nx, int ny, int nz, const double* P, double max_rho, int solid, int bb,
                             int code, int phase_id, uint8_t* mask, uint8_t* phase) {
    Grid g(nx, ny, nz, 3);
    g.put(g.lats[0], P);
    g.put8(g.lats[1], mask);
    g.put8(g.lats[2], phase);
    std::vector<uint8_t> before(mask, mask + (size_t)nx * ny * nz);
    precipNodeConversion3D<double, CaStubD3Q7> p(nx, ny, nz, max_rho, solid, bb, code, phase_id);
    std::vector<Lat*> v = {g.lats[0], g.lats[1]};
    if (phase_id > 0) v.push_back(g.lats[2]);
    p.process(g.box(), v);
    g.get8(g.lats[1], mask);
    g.get8(g.lats[2], phase);
    long long changed = 0;
    for (size_t n = 0; n < before.size(); ++n) changed += before[n] != mask[n];
    return changed;
}

/* dissolNodeConversion3D on [C.., mask, phase] */
long long ref_dissol_convert(int nx, int ny, int nz, int S, const double* C, int pore0, int solid, int bb,
                             int n_phases, const int* ids, const int* materials, const int* substrates,
                             const double* full, const int* is_precip, double reopen,
                             uint8_t* mask, uint8_t* phase) {
    const size_t N = (size_t)nx * ny * nz;
    Grid g(nx, ny, nz, (size_t)S + 2);
    for (int s = 0; s < S; ++s) g.put(g.lats[s], C + s * N);
    g.put8(g.lats[S], mask);
    g.put8(g.lats[S + 1], phase);
    std::vector<uint8_t> before(mask, mask + N);
    DissolutionConfig dcfg = dissol_config(n_phases, ids, materials, substrates, full, is_precip, reopen, 1);
    dissolNodeConversion3D<double, CaStubD3Q7> d(S, pore0, solid, bb, &dcfg);
    d.process(g.box(), g.lats);
    g.get8(g.lats[S], mask);
    g.get8(g.lats[S + 1], phase);
    long long changed = 0;
    for (size_t n = 0; n < N; ++n) changed += before[n] != mask[n];
    return changed;
}

}  // extern "C"
