/*
 * zhao_harness.cpp -- the reference's default rate laws (the Zhao network of
 * defineKinetics.hh and defineAbioticKinetics.hh at the reference root),
 * compiled from the reference tree against plb_stub.h (oracle/Makefile), with
 * C entry points over plain arrays.  Test infrastructure only: it pins the
 * library's span restatement of the same laws (include/complab_ratelaw.hpp).
 *
 *   ref_zhao_kinetics  defineRxnKinetics(B, C, subsR, bioR, mask)
 *   ref_zhao_abiotic   defineAbioticRxnKinetics(C, subsR, mask)
 */
#include "plb_stub.h"
#include "defineKinetics.hh"
#include "defineAbioticKinetics.hh"

extern "C" void ref_zhao_kinetics(const double* B, int nB, const double* C, int nC, double* subsR, double* bioR,
                                  int mask) {
    std::vector<double> b(B, B + nB), c(C, C + nC), s(nC, 0.0), r(nB, 0.0);
    defineRxnKinetics(b, c, s, r, (plint)mask);
    for (int i = 0; i < nC; ++i) subsR[i] = s[i];
    for (int i = 0; i < nB; ++i) bioR[i] = r[i];
}

extern "C" void ref_zhao_abiotic(const double* C, int nC, double* subsR, int mask) {
    std::vector<double> c(C, C + nC), s(nC, 0.0);
    defineAbioticRxnKinetics(c, s, (plint)mask);
    for (int i = 0; i < nC; ++i) subsR[i] = s[i];
}
