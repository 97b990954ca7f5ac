/*
 * ratelaw_host.cpp -- the library's compiled rate laws
 * (include/complab_ratelaw.hpp) built for the host with g++, with C entry
 * points over plain arrays.  Test infrastructure: the CPU tests compare these
 * with the reference's own headers (oracle/ref/zhao_harness.cpp), and the
 * oracle's transport step calls them as its rate law when a test runs a
 * compiled chemistry on the GPU.
 */
#include "../include/complab_ratelaw.hpp"

extern "C" void port_zhao_kinetics(const double* B, int nB, const double* C, int nC, double* subsR, double* bioR,
                                   int mask) {
    clrl::zhao::kinetics(clrl::cspan{B, nB}, clrl::cspan{C, nC}, clrl::dspan{subsR, nC}, clrl::dspan{bioR, nB}, mask);
}

extern "C" void port_zhao_abiotic(const double* C, int nC, double* subsR, int mask) {
    clrl::zhao::abiotic(clrl::cspan{C, nC}, clrl::dspan{subsR, nC}, mask);
}
