/*
 * ref_harness.cpp -- extern "C" entry points over the reference's own
 * Palabos-free code, compiled from the reference tree (paths given by the
 * build recipe oracle/Makefile).  Test infrastructure only: it pins the FP64
 * oracle (oracle.c) and the CUDA path against the reference's arithmetic.
 *
 *   ref_pcf_solve      EquilibriumChemistry<T>::calculate_species_concentrations
 *                      (src/complab3d_processors_part4_eqsolver.hh:1187-1214), the
 *                      live PCF + Anderson solver, with the settings of
 *                      src/complab.cpp:417-426 (max 200 iterations, tol 1e-10,
 *                      Anderson depth 4).
 *   ref_surrogate      defineSurrogateModel (surrogateModel.hh:252-501), the shipped
 *                      2->10->10->10->10->1 network.
 *   ref_kinetics_ex05  defineRxnKinetics of examples/05_biotic_cellular_automaton.
 *   ref_abiotic_ex13   defineAbioticRxnKinetics of examples/13_precipitation.
 */
#include "plb_stub.h"
#include <cstdint>
#include <cstring>
#include "src/complab3d_processors_part4_eqsolver.hh"
#include "surrogateModel.hh"
namespace ex05 {
#include "examples/05_biotic_cellular_automaton/defineKinetics.hh"
}
namespace ex13 {
#include "examples/13_precipitation/defineAbioticKinetics.hh"
}

extern "C" {

/* species: n x ns input concentrations; out: n x ns; conv/iters per solve */
int ref_pcf_solve(int nc, int ns, const double* stoich /*ns x nc*/, const double* logk,
                  const int* comp_species, const double* species, double* out,
                  int32_t* iters, uint8_t* conv, int64_t n, int max_iter, double tol, int depth)
{
    EquilibriumChemistry<double> eq;
    std::vector<std::string> sn(ns), cn(nc);
    for (int i = 0; i < ns; ++i) sn[i] = "S" + std::to_string(i);
    for (int j = 0; j < nc; ++j)
        cn[j] = (comp_species[j] >= 0) ? sn[comp_species[j]] : ("C" + std::to_string(j));
    eq.setSpeciesNames(sn);
    eq.setComponentNames(cn);
    std::vector<double> lk(logk, logk + ns);
    eq.setLogK(lk);
    std::vector<std::vector<double>> S(ns, std::vector<double>(nc));
    for (int i = 0; i < ns; ++i) for (int j = 0; j < nc; ++j) S[i][j] = stoich[i*nc + j];
    eq.setStoichiometryMatrix(S);
    eq.setMaxIterations(max_iter);
    eq.setTolerance(tol);
    eq.setAndersonDepth(depth);
    for (int64_t k = 0; k < n; ++k) {
        std::vector<double> c(species + k*ns, species + (k+1)*ns);
        std::vector<double> r = eq.calculate_species_concentrations(c);
        for (int i = 0; i < ns; ++i) out[k*ns + i] = r[i];
        if (iters) iters[k] = (int32_t)eq.getLastIterations();
        if (conv) conv[k] = eq.didConverge() ? 1 : 0;
    }
    return 0;
}

/* Fin: n x 2 (mmol/gDW/h); bioR out: n */
int ref_surrogate(const double* fin, double* bior, int64_t n)
{
    for (int64_t k = 0; k < n; ++k) {
        std::vector<std::vector<double>> Fin(1, std::vector<double>(2)), Fout;
        Fin[0][0] = fin[2*k]; Fin[0][1] = fin[2*k + 1];
        Fout = Fin;
        std::vector<double> bioR(1, 0.0);
        defineSurrogateModel(0, Fin, Fout, bioR, 2);
        bior[k] = bioR[0];
    }
    return 0;
}

int ref_kinetics_ex05(const double* B, int nb, const double* C, int nc, int mask,
                      double* subsR, double* bioR)
{
    std::vector<double> b(B, B + nb), c(C, C + nc), sr(nc, 0.0), br(nb, 0.0);
    ex05::defineRxnKinetics(b, c, sr, br, mask);
    for (int i = 0; i < nc; ++i) subsR[i] = sr[i];
    for (int i = 0; i < nb; ++i) bioR[i] = br[i];
    return 0;
}

int ref_abiotic_ex13(const double* C, int nc, int mask, double* subsR)
{
    std::vector<double> c(C, C + nc), sr(nc, 0.0);
    ex13::defineAbioticRxnKinetics(c, sr, mask);
    for (int i = 0; i < nc; ++i) subsR[i] = sr[i];
    return 0;
}

}
