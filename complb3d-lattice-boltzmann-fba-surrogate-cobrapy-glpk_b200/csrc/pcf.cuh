// pcf.cuh -- the reference's live speciation solver on the device: positive
// continued fractions (PCF) with Anderson acceleration, one solve per thread.
//
// Restates EquilibriumChemistry<T> (src/complab3d_processors_part4_eqsolver.hh):
//   calc_species (:442-496), calc_reactive_product_sums (:540-640),
//   pcf_residual (:664-726), qr_decomposition (:817-868),
//   solve_upper_triangular (:887-904), solve_equilibrium_anderson (:952-1172).
// Unknowns x_j = log10 of the free components.  Each iteration evaluates every
// species, splits each component's mass balance into the species carrying it
// with a positive coefficient (S_R) and the total plus those carrying it with a
// negative one (S_P), and takes the correction f_j = log10(S_P/S_R)/mu_min_j
// (clamped to +-10, 0 for an absent component); convergence is ||f||_2 < tol.
// From the second iteration the step is Anderson's: the least-squares
// combination of the last `depth` correction differences (classical
// Gram-Schmidt QR, oldest columns dropped while the diagonal ratio exceeds
// 1e10), mixing 1.  Sums and products are rounded one operation at a time
// (no fused multiply-add), as the reference's x86-64 build computes them;
// exp10 / log10 are CUDA's, so iterates can differ from the reference's in the
// last bits and a solve that ends near the tolerance can take one iteration
// more or less.  The iteration history lives in local memory.
#pragma once
#include "newton.cuh"

namespace cl {

constexpr int kPcfMaxDepth = 8;   // anderson_depth accepted by the device solver

// std::min / std::max as the reference calls them: a NaN first argument passes
__device__ __forceinline__ double pcf_min(double a, double b) { return (b < a) ? b : a; }
__device__ __forceinline__ double pcf_max(double a, double b) { return (a < b) ? b : a; }

// calc_species for equilibrium species i; init is its input concentration
template <int NC>
__device__ __forceinline__ double pcf_species(const EqDev& e, int i, const double* x, double init) {
    double lc = e.logk[i];
#pragma unroll
    for (int j = 0; j < NC; ++j) lc = __dadd_rn(lc, __dmul_rn(e.stoich[i][j], x[j]));
    lc = pcf_max(pcf_min(lc, 1.0), -30.0);
    double v = exp10(lc);
    if (isnan(v) || isinf(v)) v = init > 1e-30 ? init : 1e-30;
    return pcf_max(pcf_min(v, 10.0), 1e-30);
}

// a species that takes no part in the equilibrium keeps its input (clamped)
__device__ __forceinline__ double pcf_passive(double init) { return init > 1e-30 ? pcf_min(init, 10.0) : 1e-30; }

// the PCF correction f at x; init(i) = input species i (init[i * istride])
template <int NC>
__device__ void pcf_correction(const EqDev& e, const double* T, const double* x, const double* init, int istride,
                               double* f) {
    double pos[NC], neg[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) { pos[j] = 0.0; neg[j] = 0.0; }
    for (int i = 0; i < e.ns; ++i) {
        if (!e.active[i]) continue;
        const double c = pcf_max(pcf_species<NC>(e, i, x, init[i * istride]), 1e-30);
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            const double mu = e.stoich[i][j];
            if (mu > 1e-15) pos[j] = __dadd_rn(pos[j], __dmul_rn(mu, c));
            else if (mu < -1e-15) neg[j] = __dadd_rn(neg[j], __dmul_rn(fabs(mu), c));
        }
    }
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        double sr, sp;
        if (T[j] >= 0.0) { sr = pos[j]; sp = __dadd_rn(T[j], neg[j]); }
        else { sr = __dadd_rn(fabs(T[j]), pos[j]); sp = neg[j]; }
        sr = pcf_max(sr, 1e-30);
        sp = pcf_max(sp, 1e-30);
        double v = __dmul_rn(e.inv_mu[j], __dsub_rn(log10(sp), log10(sr)));
        v = pcf_max(pcf_min(v, 10.0), -10.0);
        if (isnan(v) || isinf(v)) v = 0.0;
        if (T[j] <= 1e-18) v = 0.0;
        f[j] = v;
    }
}

template <int NC>
__device__ __forceinline__ double pcf_norm(const double* v) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < NC; ++k) s = __dadd_rn(s, __dmul_rn(v[k], v[k]));
    return __dsqrt_rn(s);
}

// classical Gram-Schmidt of the columns cols[c0 .. c0+m-1]; R upper triangle
template <int NC>
__device__ void pcf_qr(double (*cols)[NC], int c0, int m, double (*Q)[NC], double (*R)[kPcfMaxDepth],
                       double* cond) {
    double rmax = 0.0, rmin = 1.7976931348623157e308;
    for (int j = 0; j < m; ++j) {
#pragma unroll
        for (int k = 0; k < NC; ++k) Q[j][k] = cols[c0 + j][k];
        for (int i = 0; i < j; ++i) {
            double d = 0.0;
#pragma unroll
            for (int k = 0; k < NC; ++k) d = __dadd_rn(d, __dmul_rn(Q[i][k], cols[c0 + j][k]));
            R[i][j] = d;
#pragma unroll
            for (int k = 0; k < NC; ++k) Q[j][k] = __dsub_rn(Q[j][k], __dmul_rn(d, Q[i][k]));
        }
        const double rjj = pcf_norm<NC>(Q[j]);
        R[j][j] = rjj;
        if (rjj > 1e-15) {
#pragma unroll
            for (int k = 0; k < NC; ++k) Q[j][k] = __ddiv_rn(Q[j][k], rjj);
        }
        const double a = fabs(rjj);
        if (a > rmax) rmax = a;
        if (a > 1e-30 && a < rmin) rmin = a;
    }
    *cond = m == 0 ? 1.0 : (rmin > 1e-30 ? __ddiv_rn(rmax, rmin) : 1.7976931348623157e308);
}

// solve_equilibrium_anderson from x (the cold start) with totals T; on return
// x holds the last iterate.  Returns getLastIterations(); *conv = didConverge().
template <int NC>
__device__ int eq_pcf(const EqDev& e, const double* T, const double* init, int istride, double* x, int max_iter,
                      double tol, int depth, int* conv) {
    double hx[kPcfMaxDepth + 2][NC], hf[kPcfMaxDepth + 2][NC];    // history, oldest first
    double f[NC], xn[NC];
    *conv = 0;
    pcf_correction<NC>(e, T, x, init, istride, f);
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        hx[0][j] = x[j];
        hf[0][j] = f[j];
        x[j] = pcf_max(pcf_min(__dadd_rn(x[j], f[j]), 1.0), -30.0);
    }
    int hn = 1, iters = 0;
    for (int it = 1; it < max_iter; ++it) {
        iters = it;
        pcf_correction<NC>(e, T, x, init, istride, f);
        if (pcf_norm<NC>(f) < tol) { *conv = 1; break; }
#pragma unroll
        for (int j = 0; j < NC; ++j) { hx[hn][j] = x[j]; hf[hn][j] = f[j]; }
        ++hn;
        const int m = hn - 1 < depth ? hn - 1 : depth;
        double dF[kPcfMaxDepth][NC], dX[kPcfMaxDepth][NC], Q[kPcfMaxDepth][NC], R[kPcfMaxDepth][kPcfMaxDepth];
        for (int i = 0; i < m; ++i) {
            const int a = hn - m - 1 + i;
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                dF[i][j] = __dsub_rn(hf[a + 1][j], hf[a][j]);
                dX[i][j] = __dsub_rn(hx[a + 1][j], hx[a][j]);
            }
        }
        double cond;
        int first = 0;                       // oldest columns dropped
        pcf_qr<NC>(dF, 0, m, Q, R, &cond);
        while (cond > 1e10 && m - first > 1) {
            ++first;
            pcf_qr<NC>(dF, first, m - first, Q, R, &cond);
        }
        const int mm = m - first;
        double g[kPcfMaxDepth];
        for (int i = mm - 1; i >= 0; --i) {
            double v = 0.0;
#pragma unroll
            for (int k = 0; k < NC; ++k) v = __dadd_rn(v, __dmul_rn(Q[i][k], f[k]));
            for (int k = i + 1; k < mm; ++k) v = __dsub_rn(v, __dmul_rn(R[i][k], g[k]));
            if (fabs(R[i][i]) > 1e-30) v = __ddiv_rn(v, R[i][i]);
            g[i] = v;
        }
        double sx[NC], sf[NC];
#pragma unroll
        for (int j = 0; j < NC; ++j) { sx[j] = 0.0; sf[j] = 0.0; }
        for (int i = 0; i < mm; ++i) {
#pragma unroll
            for (int j = 0; j < NC; ++j) {
                sx[j] = __dadd_rn(sx[j], __dmul_rn(dX[first + i][j], g[i]));
                sf[j] = __dadd_rn(sf[j], __dmul_rn(dF[first + i][j], g[i]));
            }
        }
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            xn[j] = __dadd_rn(__dsub_rn(x[j], sx[j]), __dsub_rn(f[j], sf[j]));
            double v = pcf_max(pcf_min(xn[j], 1.0), -30.0);
            if (isnan(v) || isinf(v)) v = x[j];
            x[j] = v;
        }
        // keep the depth + 1 newest entries
        while (hn > depth + 1) {
            for (int a = 1; a < hn; ++a) {
#pragma unroll
                for (int j = 0; j < NC; ++j) { hx[a - 1][j] = hx[a][j]; hf[a - 1][j] = hf[a][j]; }
            }
            --hn;
        }
    }
    return iters;
}

// component totals of the species (calc_component_totals) and the cold start
template <int NC>
__device__ __forceinline__ void pcf_totals_and_start(const EqDev& e, const double* c, int stride, double* T,
                                                     double* x) {
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        double t = 0.0;
        for (int i = 0; i < e.ns; ++i) {
            if (!e.active[i]) continue;
            t = __dadd_rn(t, __dmul_rn(e.stoich[i][j], pcf_max(pcf_min(c[i * stride], 10.0), 1e-30)));
        }
        T[j] = pcf_max(t, 1e-30);
        const int idx = e.comp_species[j];
        const double cj = (idx >= 0 && idx < e.ns) ? c[idx * stride] : 1e-7;
        x[j] = log10(pcf_max(pcf_min(cj, 10.0), 1e-30));
    }
}

}  // namespace cl
