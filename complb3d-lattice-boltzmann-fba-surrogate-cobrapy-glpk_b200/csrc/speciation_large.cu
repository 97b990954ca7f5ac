// speciation_large.cu -- batch Newton speciation for large tableaux.
//
// The transport step and the small-tableau batch solver keep a voxel's
// Newton state in one thread's registers, which holds up to five
// components.  Field tableaux are larger: the reference ships a uranium
// network of 17 components over 95 species
// (CompLaB_example_uranium_zhao.xml, the <equilibrium> block).  Here one warp
// solves one system:
//   - the block stages the tableau once in shared memory, transposed
//     (component-major), so lane a streams its component's column;
//   - species: the lanes split the species (i = lane, lane + 32, ...), each
//     writing c_i = 10^(logK_i + sum_j S_ij x_j) (clamped to [1e-30, 10]) and
//     its Jacobian weight into the warp's shared arrays;
//   - rows: lane a < n_comp forms F_a = sum_i S_ia c_i - T_a, the scale
//     sum_i |S_ia| c_i and row a of J = ln10 S^T diag(c) S, summing over the
//     species in order (the order of the one-thread solver);
//   - Cholesky of J right-looking over the columns, lanes on the rows; the two
//     triangular solves on lane 0.
// The iteration is the one of newton.cuh (relative mass-balance residual,
// clamped species out of J, 2-decade step cap, Armijo backtracking on the
// weighted residual with at most 40 halvings, a solve stops when every trial
// fails), so the solutions agree with the small solver and the FP64 oracle
// to the residual tolerance.
#include "internal.h"
#include "speciation_large.h"
#include "newton.cuh"

namespace cl {

constexpr int kLgWarps = 4;

struct LgWarp {
    double x[CL_MAX_COMP], T[CL_MAX_COMP], F[CL_MAX_COMP], Ft[CL_MAX_COMP], sc[CL_MAX_COMP], w[CL_MAX_COMP];
    double d[CL_MAX_COMP], xt[CL_MAX_COMP], Li[CL_MAX_COMP];
    double L[CL_MAX_COMP][CL_MAX_COMP + 1];
    double c[CL_MAX_SPECIES], cj[CL_MAX_SPECIES];
};

__device__ __forceinline__ double lg_max_nan(double a, double b) {
    return (a != a || b != b) ? (a + b) : fmax(a, b);
}
__device__ __forceinline__ double lg_warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = lg_max_nan(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double lg_warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// species of the point xs into W.c / W.cj (cj: zero for a clamped species)
__device__ __forceinline__ void lg_species(const LgTableau& e, const double* St, const double* lk,
                                           const uint8_t* act, const double* xs, LgWarp& W, int lane) {
    for (int i = lane; i < e.ns; i += 32) {
        double c = 0.0, cj = 0.0;
        if (act[i]) {
            double lc = lk[i];
            for (int j = 0; j < e.nc; ++j) lc = fma(St[j * e.ns + i], xs[j], lc);
            if (lc > 1.0) c = 10.0;
            else if (lc < -30.0) c = 1e-30;
            else { c = cl_exp10(lc); cj = c; }
        }
        W.c[i] = c;
        W.cj[i] = cj;
    }
    __syncwarp();
}

// row a = lane of F (into Fo) and, with want_J, the scales and the lower
// triangle of J; returns the warp's relative residual max_a |F_a| / sc_a
__device__ __forceinline__ double lg_rows(const LgTableau& e, const double* St, LgWarp& W, double* Fo, bool want_J,
                                          int lane) {
    double r = 0.0;
    if (lane < e.nc) {
        const double* Sa = St + lane * e.ns;
        double f = -W.T[lane], s = 0.0;
        for (int i = 0; i < e.ns; ++i) {
            const double sa = Sa[i];
            f = fma(sa, W.c[i], f);
            s = fma(fabs(sa), W.c[i], s);
        }
        Fo[lane] = f;
        if (want_J) {
            W.sc[lane] = s;
            for (int b = 0; b <= lane; ++b) {
                const double* Sb = St + b * e.ns;
                double acc = 0.0;
                for (int i = 0; i < e.ns; ++i) acc = fma(Sa[i] * W.cj[i], Sb[i], acc);
                W.L[lane][b] = acc;
            }
        }
        r = fabs(f) / fmax(s, 1e-300);
    }
    __syncwarp();
    return lg_warp_max(r);
}

// weighted norm ||F_a w_a||_2 over the components
__device__ __forceinline__ double lg_norm(const LgTableau& e, const LgWarp& W, const double* Fv, int lane) {
    double q = 0.0;
    if (lane < e.nc) { const double r = Fv[lane] * W.w[lane]; q = r * r; }
    return sqrt(lg_warp_sum(q));
}

// Newton from W.x with at most max_iter iterations; returns the iterations,
// *conv = 1 at the residual tolerance
__device__ int lg_newton(const LgTableau& e, const double* St, const double* lk, const uint8_t* act, LgWarp& W,
                         int max_iter, double tol, int* conv, int lane) {
    const double ln10 = 2.302585092994046;
    const int nc = e.nc;
    *conv = 0;
    bool stuck = false;
    for (int it = 0; it < max_iter; ++it) {
        lg_species(e, St, lk, act, W.x, W, lane);
        const double rel = lg_rows(e, St, W, W.F, true, lane);
        if (lane < nc) W.w[lane] = 1.0 / fmax(W.sc[lane], 1e-300);
        __syncwarp();
        if (rel <= tol) { *conv = 1; return it; }
        if (!(rel < 1e300) || stuck) return it;
        const double fn = lg_norm(e, W, W.F, lane);
        // Cholesky of ln10 J, right-looking; L[a][k] below the diagonal, Li the
        // reciprocal square roots of the pivots
        if (lane < nc)
            for (int b = 0; b <= lane; ++b) W.L[lane][b] *= ln10;
        __syncwarp();
        bool ok = true;
        for (int k = 0; k < nc; ++k) {
            const double dkk = W.L[k][k];
            if (!(dkk > 1e-300)) { ok = false; break; }
            const double lik = rsqrt(dkk);
            if (lane == 0) W.Li[k] = lik;
            if (lane > k && lane < nc) W.L[lane][k] *= lik;
            __syncwarp();
            if (lane > k && lane < nc)
                for (int b = k + 1; b <= lane; ++b) W.L[lane][b] -= W.L[lane][k] * W.L[b][k];
            __syncwarp();
        }
        if (!ok) return it + 1;
        if (lane == 0) {
            for (int a = 0; a < nc; ++a) {
                double s = -W.F[a];
                for (int k = 0; k < a; ++k) s -= W.L[a][k] * W.d[k];
                W.d[a] = s * W.Li[a];
            }
            for (int a = nc - 1; a >= 0; --a) {
                double s = W.d[a];
                for (int k = a + 1; k < nc; ++k) s -= W.L[k][a] * W.d[k];
                W.d[a] = s * W.Li[a];
            }
            double dmax = 0.0;
            for (int a = 0; a < nc; ++a) dmax = fmax(dmax, fabs(W.d[a]));
            if (dmax > 2.0) {
                const double sfac = 2.0 / dmax;
                for (int a = 0; a < nc; ++a) W.d[a] *= sfac;
            }
        }
        __syncwarp();
        double alpha = 1.0;
        bool accepted = false;
        for (int ls = 0; ls < 40; ++ls) {
            if (lane < nc) W.xt[lane] = fmin(fmax(fma(alpha, W.d[lane], W.x[lane]), -30.0), 1.0);
            __syncwarp();
            lg_species(e, St, lk, act, W.xt, W, lane);
            lg_rows(e, St, W, W.Ft, false, lane);
            const double fnt = lg_norm(e, W, W.Ft, lane);
            if (fnt < fn * (1.0 - 1e-4 * alpha)) { accepted = true; break; }
            if (alpha < 1e-15) break;
            alpha *= 0.5;
        }
        if (lane < nc) W.x[lane] = W.xt[lane];
        __syncwarp();
        stuck = !accepted;
    }
    lg_species(e, St, lk, act, W.x, W, lane);
    const double rel = lg_rows(e, St, W, W.Ft, false, lane);
    if (rel <= tol) *conv = 1;
    return max_iter;
}

// one warp per system: start (cold: the reference's rule from the species
// vector; given: x_io), then, with a given start and species vectors, the cold
// start after warm_iter iterations
__global__ void __launch_bounds__(32 * kLgWarps) eq_large_kernel(LgTableau e, const double* __restrict__ totals,
                                                                 const double* __restrict__ cold_species,
                                                                 double* x_io, int32_t* iters, uint8_t* status,
                                                                 int64_t n, int start, int max_iter, int warm_iter,
                                                                 double tol, unsigned long long* nonconv) {
    extern __shared__ double lg_smem[];
    double* St = lg_smem;                                   // nc x ns, component-major
    double* lk = St + e.nc * e.ns;                          // ns
    LgWarp* Wall = reinterpret_cast<LgWarp*>(lk + e.ns);    // kLgWarps
    uint8_t* act = reinterpret_cast<uint8_t*>(Wall + kLgWarps);
    for (int q = threadIdx.x; q < e.nc * e.ns; q += blockDim.x) {
        const int j = q / e.ns, i = q - j * e.ns;
        St[q] = e.stoich[(int64_t)i * e.nc + j];
    }
    for (int i = threadIdx.x; i < e.ns; i += blockDim.x) { lk[i] = e.logk[i]; act[i] = e.active[i]; }
    __syncthreads();
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    LgWarp& W = Wall[wid];
    unsigned long long miss = 0;
    const bool fallback = start == CL_EQ_START_GIVEN && cold_species != nullptr;
    for (int64_t v = (int64_t)blockIdx.x * kLgWarps + wid; v < n; v += (int64_t)gridDim.x * kLgWarps) {
        if (lane < e.nc) W.T[lane] = totals[v * e.nc + lane];
        int total_it = 0, conv = 0, st = 2;
        for (int phase = (start == CL_EQ_START_COLD) ? 1 : 0; phase < 2; ++phase) {
            if (lane < e.nc) {
                if (phase == 0) W.x[lane] = x_io[v * e.nc + lane];
                else {
                    double c = 1e-7;
                    const int idx = e.comp_species[lane];
                    if (idx >= 0) c = cold_species[v * e.ns + idx];
                    W.x[lane] = log10(fmin(fmax(c, 1e-30), 10.0));
                }
            }
            __syncwarp();
            const int budget = (phase == 0 && fallback) ? warm_iter : max_iter;
            total_it += lg_newton(e, St, lk, act, W, budget, tol, &conv, lane);
            if (conv) { st = (phase == 0 || start == CL_EQ_START_COLD) ? 0 : 1; break; }
            if (phase == 0 && !fallback) break;
        }
        if (lane < e.nc) x_io[v * e.nc + lane] = W.x[lane];
        if (lane == 0) {
            if (iters) iters[v] = total_it;
            if (status) status[v] = (uint8_t)st;
            miss += conv ? 0 : 1;
        }
        __syncwarp();
    }
    if (lane == 0 && miss) atomicAdd(nonconv, miss);
}

size_t lg_smem_bytes(int nc, int ns) {
    return sizeof(double) * ((size_t)nc * ns + ns) + sizeof(LgWarp) * kLgWarps + (size_t)ns + 16;
}

int lg_solve(const LgTableau& e, cudaStream_t stream, const double* d_totals, const double* d_cold, double* d_x,
             int32_t* d_iters, uint8_t* d_status, int64_t n, int start, int max_iter, int warm_iter, double tol,
             unsigned long long* d_count) {
    const size_t smem = lg_smem_bytes(e.nc, e.ns);
    CL_CUDA(cudaFuncSetAttribute(eq_large_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CL_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), stream));
    const int blocks = grid_for((n + kLgWarps - 1) / kLgWarps, 1, 148 * 4);
    eq_large_kernel<<<blocks, 32 * kLgWarps, smem, stream>>>(e, d_totals, d_cold, d_x, d_iters, d_status, n, start,
                                                             max_iter, warm_iter, tol, d_count);
    CL_LAUNCH_CHECK("eq_large_kernel");
    unsigned long long miss = 0;
    CL_CUDA(cudaMemcpyAsync(&miss, d_count, sizeof miss, cudaMemcpyDeviceToHost, stream));
    CL_CUDA(cudaStreamSynchronize(stream));
    return miss ? CL_WARN_NOT_CONVERGED : CL_OK;
}

}  // namespace cl
