// speciation_large.h -- the warp-per-system Newton solver for tableaux larger
// than the one-thread solver holds (speciation_large.cu).
#pragma once
#include "internal.h"

namespace cl {

// a tableau in device memory: stoich n_species x n_comp (row-major), logK and
// the active flags (species with any nonzero coefficient) per species
struct LgTableau {
    int nc, ns;
    const double* stoich;
    const double* logk;
    const uint8_t* active;
    int comp_species[CL_MAX_COMP];
};

size_t lg_smem_bytes(int nc, int ns);
// statuses: 0 converged from the first start, 1 after the cold fallback, 2 not converged
int lg_solve(const LgTableau& e, cudaStream_t stream, const double* d_totals, const double* d_cold, double* d_x,
             int32_t* d_iters, uint8_t* d_status, int64_t n, int start, int max_iter, int warm_iter, double tol,
             unsigned long long* d_count);

}  // namespace cl
