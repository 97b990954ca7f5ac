// newton.cuh -- FP64 Newton speciation for one voxel per thread.
//
// Restates the Newton-Raphson reserve solver of the reference
// (src/complab3d_processors_part4_eqsolver_NR_reserve.hh:512-615):
//   unknowns x_j = log10 of the free component concentrations,
//   c_i = 10^(logK_i + sum_j S_ij x_j) clamped to [1e-30, 10]   (calc_species, :442-496 of the live solver)
//   F_j = sum_i S_ij c_i - T_j                                  (calc_residual, :309-328)
//   J   = ln10 * S^T diag(c) S                                  (calc_jacobian, :356-377)
//   J d = -F, Armijo backtracking on ||F||_2, alpha halving, <= 40 trials (:577-598)
// The linear solve is a Cholesky factorisation (J is symmetric positive
// definite); the reserve uses Gaussian elimination with partial pivoting, which
// gives the same step up to rounding.  Deviations from the reserve, shared with
// the FP64 oracle (without them the reserve stalls on most cold starts of the
// 5x14 random tableaux):
//   - convergence: relative mass-balance residual max_j |F_j| / sum_i |S_ij| c_i <= tol;
//   - species at a clamp bound contribute nothing to J;
//   - the step is scaled so that no component moves more than 2 decades;
//   - the Armijo merit is ||F_j / sum_i |S_ij| c_i||_2 with the current weights
//     (its test compared in squares);
//   - a solve whose 40 backtracking trials all fail stops (the next iterate
//     would be the same point to ~1e-12 of a step).
// Species are evaluated on the fly (no per-species storage), the component
// count NC is a template parameter so every array lives in registers.
#pragma once
#include <cmath>
#include "../../include/complab_gpu.h"

namespace cl {

// the one-thread solvers' tableau: up to kEqDevSpecies species (one per
// solute in the transport step) over up to kEqDevComp components (five are
// instantiated); larger tableaux go to the warp solver (speciation_large.cu)
constexpr int kEqDevSpecies = CL_MAX_SOLUTES, kEqDevComp = 8;
struct EqDev {
    int ns;
    int all_int;                       // every stoichiometric coefficient is an integer in [-8, 8]
    double stoich[kEqDevSpecies][kEqDevComp];
    double absS[kEqDevSpecies][kEqDevComp];
    double logk[kEqDevSpecies];
    double k10[kEqDevSpecies];         // 10^logK
    signed char ipow[kEqDevSpecies][kEqDevComp];
    int active[kEqDevSpecies];
    int comp_species[kEqDevComp];
    int neg[kEqDevComp];               // some species carries component j with a negative power
    double inv_mu[kEqDevComp];         // PCF: 1 / the smallest positive coefficient of component j (at most 1)
    int solver;                        // CL_EQ_SOLVER_* of the transport step
    int depth;                         // PCF Anderson depth
};

// (callers hold n_species <= kEqDevSpecies and n_comp <= kEqDevComp)
inline void eqdev_from_system(const cl_eq_system& s, EqDev& d) {
    d.ns = s.n_species < kEqDevSpecies ? s.n_species : kEqDevSpecies;
    const int ns = d.ns, ncm = s.n_comp < kEqDevComp ? s.n_comp : kEqDevComp;
    d.all_int = 1;
    for (int i = 0; i < kEqDevSpecies; ++i) {
        int act = 0;
        for (int j = 0; j < kEqDevComp; ++j) {
            double v = (i < ns && j < ncm) ? s.stoich[i][j] : 0.0;
            d.stoich[i][j] = v;
            d.absS[i][j] = v < 0 ? -v : v;
            if (v > 1e-10 || v < -1e-10) act = 1;
            const double r = v < 0 ? -(double)(long long)(-v + 0.5) : (double)(long long)(v + 0.5);
            if (r != v || r > 8 || r < -8) d.all_int = 0;
            d.ipow[i][j] = (signed char)r;
        }
        d.active[i] = act;
        d.logk[i] = i < ns ? s.logk[i] : 0.0;
        d.k10[i] = std::pow(10.0, d.logk[i]);
    }
    for (int j = 0; j < kEqDevComp; ++j) {
        d.comp_species[j] = j < ncm ? s.comp_species[j] : -1;
        d.neg[j] = 0;
        for (int i = 0; i < ns && j < ncm; ++i) if (d.ipow[i][j] < 0) d.neg[j] = 1;
        // pcf_residual's mu_min (part4_eqsolver.hh:690-697): starts at 1, equilibrium species only
        double mu_min = 1.0;
        for (int i = 0; i < ns && j < ncm; ++i) {
            if (!d.active[i]) continue;
            const double mu = s.stoich[i][j];
            if (mu > 1e-10 && mu < mu_min) mu_min = mu;
        }
        d.inv_mu[j] = 1.0 / mu_min;
    }
    d.solver = s.solver;
    d.depth = s.anderson_depth > 0 ? s.anderson_depth : 4;
}

// The tableau a solve reads.  TabRun: the run-time tableau (EqDev).
// TabFixed<Fix>: an integer stoichiometry fixed at compile time
// (Fix::ns, Fix::coef(i, j), with the equilibrium constants still from the
// run), so that after the species and component loops unroll every zero
// coefficient, every unit power and every inactive species folds away.
struct TabRun {
    static constexpr bool kFixed = false;
    const EqDev& e;
    __device__ __forceinline__ int ns() const { return e.ns; }
    __device__ __forceinline__ bool active(int i) const { return e.active[i] != 0; }
    __device__ __forceinline__ double s(int i, int j) const { return e.stoich[i][j]; }
    __device__ __forceinline__ double abs_s(int i, int j) const { return e.absS[i][j]; }
    __device__ __forceinline__ int ipow(int i, int j) const { return e.ipow[i][j]; }
    __device__ __forceinline__ bool all_int() const { return e.all_int != 0; }
    __device__ __forceinline__ bool neg(int j) const { return e.neg[j] != 0; }
    __device__ __forceinline__ double logk(int i) const { return e.logk[i]; }
    __device__ __forceinline__ double k10(int i) const { return e.k10[i]; }
};

template <class Fix>
struct TabFixed {
    static constexpr bool kFixed = true;
    const EqDev& e;
    __device__ __forceinline__ static constexpr int ns() { return Fix::ns; }
    __device__ __forceinline__ static constexpr bool active(int i) {
        bool a = false;
        for (int j = 0; j < Fix::nc; ++j) a = a || Fix::coef(i, j) != 0;
        return a;
    }
    __device__ __forceinline__ static constexpr double s(int i, int j) { return (double)Fix::coef(i, j); }
    __device__ __forceinline__ static constexpr double abs_s(int i, int j) {
        return (double)(Fix::coef(i, j) < 0 ? -Fix::coef(i, j) : Fix::coef(i, j));
    }
    __device__ __forceinline__ static constexpr int ipow(int i, int j) { return Fix::coef(i, j); }
    __device__ __forceinline__ static constexpr bool all_int() { return true; }
    __device__ __forceinline__ static constexpr bool neg(int j) {
        bool n = false;
        for (int i = 0; i < Fix::ns; ++i) n = n || Fix::coef(i, j) < 0;
        return n;
    }
    __device__ __forceinline__ double logk(int i) const { return e.logk[i]; }
    __device__ __forceinline__ double k10(int i) const { return e.k10[i]; }
};

// 10^x in FP64 for the Newton solves, about 1 ulp: Cody-Waite argument
// reduction y = x log2(10) = n + f with n = rint(y), |f| <= 1/2, the
// product carried as an exact two-term sum (Dekker's FMA split, with the
// tail of log2(10)); 2^f = e^t, t = f ln 2, by the Taylor series to degree 13
// in Horner's form (|t| <= 0.347, truncation below 5e-18); the result scaled
// by 2^n through the exponent field.  Domain |x| < 300 (every caller clamps
// its logs to [-30, 1]); NaN gives NaN.  Measured on the coupled step it is
// 2 % faster than the library's exp10 (whose wider domain costs more).
__device__ __forceinline__ double cl_exp10(double x) {
    constexpr double kL2T = 3.321928094887362, kL2T_lo = 1.661617516973592e-16;   // log2(10) = kL2T + kL2T_lo
    constexpr double kLn2 = 0.6931471805599453, kLn2_lo = 2.3190468138462996e-17;
    const double yh = x * kL2T;
    const double yl = fma(x, kL2T, -yh) + x * kL2T_lo;
    const double n = rint(yh);
    const double f = (yh - n) + yl;                  // yh - n is exact
    const double t = fma(f, kLn2, f * kLn2_lo);
    double p = 1.0 / 6227020800.0;                   // 1/13!
    p = fma(p, t, 1.0 / 479001600.0);
    p = fma(p, t, 1.0 / 39916800.0);
    p = fma(p, t, 1.0 / 3628800.0);
    p = fma(p, t, 1.0 / 362880.0);
    p = fma(p, t, 1.0 / 40320.0);
    p = fma(p, t, 1.0 / 5040.0);
    p = fma(p, t, 1.0 / 720.0);
    p = fma(p, t, 1.0 / 120.0);
    p = fma(p, t, 1.0 / 24.0);
    p = fma(p, t, 1.0 / 6.0);
    p = fma(p, t, 1.0 / 2.0);
    p = fma(p, t, 1.0);
    p = fma(p, t, 1.0);
    const long long e = (long long)n + 1023;
    return p * __longlong_as_double(e << 52);
}

// species concentration from the component logs, clamped as calc_species
template <int NC>
__device__ __forceinline__ double species_c(const EqDev& e, int i, const double* x) {
    double lc = e.logk[i];
#pragma unroll
    for (int j = 0; j < NC; ++j) lc = fma(e.stoich[i][j], x[j], lc);
    lc = fmin(fmax(lc, -30.0), 1.0);
    return cl_exp10(lc);
}

// Free-component activities a_j = 10^x_j and their inverses, once per
// evaluation; with integer stoichiometry every species is then
// c_i = 10^logK_i * prod_j a_j^S_ij by multiplication only (NC exp10 per
// evaluation instead of one per species).  The clamp test uses the exact log.
template <int NC>
struct Powers {
    double a[NC], ai[NC];
    // inverses only of the components some species divides by
    template <class Tab>
    __device__ __forceinline__ void set(const Tab& t, const double* x) {
#pragma unroll
        for (int j = 0; j < NC; ++j) { a[j] = cl_exp10(x[j]); ai[j] = t.neg(j) ? 1.0 / a[j] : 0.0; }
    }
    __device__ __forceinline__ void set(const EqDev& e, const double* x) { set(TabRun{e}, x); }
};

template <int NC, class Tab>
__device__ __forceinline__ double species_eval(const Tab& tb, int i, const double* x, const Powers<NC>& pw,
                                               bool& clamped) {
    double lc = tb.logk(i);
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        if constexpr (Tab::kFixed) { if (tb.ipow(i, j) == 0) continue; }
        lc = fma(tb.s(i, j), x[j], lc);
    }
    if (lc > 1.0) { clamped = true; return 10.0; }
    if (lc < -30.0) { clamped = true; return 1e-30; }
    clamped = false;
    if (!tb.all_int()) return cl_exp10(lc);
    double p = tb.k10(i);
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        const int q = tb.ipow(i, j);
        if (q == 0) continue;
        const double b = q > 0 ? pw.a[j] : pw.ai[j];
        const int m = q > 0 ? q : -q;
        double t = b;
        for (int r = 1; r < m; ++r) t *= b;
        p *= t;
    }
    return p;
}

template <int NC>
__device__ __forceinline__ double species_eval(const EqDev& e, int i, const double* x, const Powers<NC>& pw,
                                               bool& clamped) {
    return species_eval<NC>(TabRun{e}, i, x, pw, clamped);
}

// F, and the relative residual
template <int NC, int NS = 0, class Tab>
__device__ __forceinline__ double eq_residual_t(const Tab& tb, const double* T, const double* x, double* F) {
    double sc[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) { F[j] = -T[j]; sc[j] = 0.0; }
    Powers<NC> pw;
    pw.set(tb, x);
#pragma unroll (NS > 0 ? NS : 1)
    for (int i = 0; i < (NS > 0 ? NS : tb.ns()); ++i) {
        if (!tb.active(i)) continue;
        bool clamped;
        const double c = species_eval<NC>(tb, i, x, pw, clamped);
#pragma unroll
        for (int j = 0; j < NC; ++j) {
            if constexpr (Tab::kFixed) { if (tb.ipow(i, j) == 0) continue; }
            F[j] = fma(tb.s(i, j), c, F[j]);
            sc[j] = fma(tb.abs_s(i, j), c, sc[j]);
        }
    }
    double rel = 0.0;
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        const double r = fabs(F[j]) / fmax(sc[j], 1e-300);
        rel = (r > rel || r != r) ? r : rel;
    }
    return rel;
}

template <int NC, int NS = 0>
__device__ __forceinline__ double eq_residual(const EqDev& e, const double* T, const double* x, double* F) {
    return eq_residual_t<NC, NS>(TabRun{e}, T, x, F);
}

// reference cold start (solve_equilibrium_anderson, part4_eqsolver.hh:977-994)
template <int NC>
__device__ __forceinline__ void eq_cold_start(const EqDev& e, const double* species, double* x) {
#pragma unroll
    for (int j = 0; j < NC; ++j) {
        double c = 1e-7;
        const int idx = e.comp_species[j];
        if (idx >= 0) c = species[idx];
        c = fmin(fmax(c, 1e-30), 10.0);
        x[j] = log10(c);
    }
}

// Runs at most max_iter Newton iterations from x.  Returns the iterations
// taken; *conv = 1 when the residual test passed.
// F = S^T c - T, sc = |S|^T c and the lower triangle of S^T diag(c) S
// (clamped species excluded) in one pass over the species
// (cbuf: where given, each equilibrium species' concentration is stored at
// cbuf[i * cstride], so a caller finds the species of the returned point)
template <int NC, int NS = 0, class Tab>
__device__ __forceinline__ void eq_eval_full(const Tab& tb, const double* T, const double* x,
                                             double* F, double* sc, double (*J)[NC], double* cbuf = nullptr,
                                             int cstride = 0) {
#pragma unroll
    for (int a = 0; a < NC; ++a) {
        F[a] = -T[a]; sc[a] = 0.0;
#pragma unroll
        for (int b = 0; b < NC; ++b) J[a][b] = 0.0;
    }
    Powers<NC> pw;
    pw.set(tb, x);
#pragma unroll (NS > 0 ? NS : 1)
    for (int i = 0; i < (NS > 0 ? NS : tb.ns()); ++i) {
        if (!tb.active(i)) continue;
        bool clamped;
        const double c = species_eval<NC>(tb, i, x, pw, clamped);
        if (cbuf) cbuf[i * cstride] = c;
        const double cj = clamped ? 0.0 : c;
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            if constexpr (Tab::kFixed) { if (tb.ipow(i, a) == 0) continue; }
            const double sa = tb.s(i, a);
            F[a] = fma(sa, c, F[a]);
            sc[a] = fma(tb.abs_s(i, a), c, sc[a]);
            const double sac = sa * cj;
#pragma unroll
            for (int b = 0; b <= a; ++b) {
                if constexpr (Tab::kFixed) { if (tb.ipow(i, b) == 0) continue; }
                J[a][b] = fma(sac, tb.s(i, b), J[a][b]);
            }
        }
    }
}

// Newton in log10 free components.  The first line-search trial (the full
// step) is evaluated with the Jacobian, which becomes the next iteration's
// when the full step is accepted (the usual case near the root); after a
// shorter step the point is evaluated again.  The iterates are the same as
// evaluating residual and Jacobian afresh at every iterate.  Returns the
// number of steps taken; *conv = 1 at the relative residual tolerance.
template <int NC, int NS = 0, class Tab>
__device__ __forceinline__ int eq_newton_reuse(const Tab& e, const double* T, double* x, int max_iter, double tol, int* conv,
                               int* stopped, double* cbuf = nullptr, int cstride = 0) {
    const double ln10 = 2.302585092994046;
    *conv = 0;
    double F[NC], sc[NC], J[NC][NC];
    eq_eval_full<NC, NS>(e, T, x, F, sc, J, cbuf, cstride);
    for (int it = 0; it < max_iter; ++it) {
        double rel = 0.0, fn = 0.0, w[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            w[a] = 1.0 / fmax(sc[a], 1e-300);
            const double r = fabs(F[a]) * w[a];
            rel = (r > rel || r != r) ? r : rel;
            fn = fma(r, r, fn);
        }
        if (rel <= tol) { *conv = 1; return it; }
        if (!(rel < 1e300)) { if (stopped) *stopped = 1; return it; }      // NaN / inf
        // fn, fnt: squared weighted residual norms (the Armijo test compares squares)
        // Cholesky of ln10*J (lower triangle), solve L L^T d = -F
        // the diagonal is kept as its reciprocal (rsqrt), so the factorisation
        // and both triangular solves multiply instead of dividing
        double L[NC][NC], Li[NC];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < NC; ++a) {
#pragma unroll
            for (int b = 0; b <= a; ++b) {
                double s = ln10 * J[a][b];
#pragma unroll
                for (int k = 0; k < b; ++k) s -= L[a][k] * L[b][k];
                if (a == b) {
                    if (!(s > 1e-300)) { ok = false; s = 1.0; }
                    Li[a] = rsqrt(s);
                } else {
                    L[a][b] = s * Li[b];
                }
            }
        }
        if (!ok) { if (stopped) *stopped = 1; return it + 1; }
        double d[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            double s = -F[a];
#pragma unroll
            for (int k = 0; k < a; ++k) s -= L[a][k] * d[k];
            d[a] = s * Li[a];
        }
#pragma unroll
        for (int a = NC - 1; a >= 0; --a) {
            double s = d[a];
#pragma unroll
            for (int k = a + 1; k < NC; ++k) s -= L[k][a] * d[k];
            d[a] = s * Li[a];
        }
        // step cap (2 decades), then Armijo backtracking on the weighted residual
        double dmax = 0.0;
#pragma unroll
        for (int a = 0; a < NC; ++a) dmax = fmax(dmax, fabs(d[a]));
        if (dmax > 2.0) {
            const double sfac = 2.0 / dmax;
#pragma unroll
            for (int a = 0; a < NC; ++a) d[a] *= sfac;
        }
        double xt[NC], Ft[NC], sct[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) xt[a] = fmin(fmax(d[a] + x[a], -30.0), 1.0);
        eq_eval_full<NC, NS>(e, T, xt, Ft, sct, J, cbuf, cstride);   // J is free once L is formed
        double fnt = 0.0;
#pragma unroll
        for (int a = 0; a < NC; ++a) { const double r = Ft[a] * w[a]; fnt = fma(r, r, fnt); }
        if (fnt < fn * ((1.0 - 1e-4) * (1.0 - 1e-4))) {
#pragma unroll
            for (int a = 0; a < NC; ++a) { x[a] = xt[a]; F[a] = Ft[a]; sc[a] = sct[a]; }
            continue;
        }
        double alpha = 0.5;
        bool accepted = false;
        for (int ls = 1; ls < 40; ++ls) {
#pragma unroll
            for (int a = 0; a < NC; ++a) xt[a] = fmin(fmax(fma(alpha, d[a], x[a]), -30.0), 1.0);
            eq_residual_t<NC, NS>(e, T, xt, Ft);
            fnt = 0.0;
#pragma unroll
            for (int a = 0; a < NC; ++a) { const double r = Ft[a] * w[a]; fnt = fma(r, r, fnt); }
            const double q = 1.0 - 1e-4 * alpha;
            if (fnt < fn * (q * q)) { accepted = true; break; }
            if (alpha < 1e-15) break;
            alpha *= 0.5;
        }
#pragma unroll
        for (int a = 0; a < NC; ++a) x[a] = xt[a];
        eq_eval_full<NC, NS>(e, T, x, F, sc, J, cbuf, cstride);
        if (!accepted) {
            // every trial failed: the next iterate is this point to ~1e-12 of
            // a step and fails the same way, so the solve stops here
            double rel2 = 0.0;
#pragma unroll
            for (int a = 0; a < NC; ++a) {
                const double r = fabs(F[a]) / fmax(sc[a], 1e-300);
                rel2 = (r > rel2 || r != r) ? r : rel2;
            }
            if (rel2 <= tol) *conv = 1;
            if (stopped) *stopped = 1;
            return it + 1;
        }
    }
    double rel = 0.0;
#pragma unroll
    for (int a = 0; a < NC; ++a) {
        const double r = fabs(F[a]) / fmax(sc[a], 1e-300);
        rel = (r > rel || r != r) ? r : rel;
    }
    if (rel <= tol) *conv = 1;
    return max_iter;
}

// The same iteration with residual and Jacobian evaluated afresh at every
// iterate (fewer live registers; used above three components).
template <int NC, int NS = 0, class Tab>
__device__ __forceinline__ int eq_newton_plain(const Tab& tb, const double* T, double* x, int max_iter, double tol, int* conv,
                               int* stopped) {
    const double ln10 = 2.302585092994046;
    *conv = 0;
    bool stuck = false;
    for (int it = 0; it < max_iter; ++it) {
        // residual and Jacobian in one pass over the species
        double F[NC], sc[NC], J[NC][NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            F[a] = -T[a]; sc[a] = 0.0;
#pragma unroll
            for (int b = 0; b < NC; ++b) J[a][b] = 0.0;
        }
        Powers<NC> pw;
        pw.set(tb, x);
#pragma unroll (NS > 0 ? NS : 1)
        for (int i = 0; i < (NS > 0 ? NS : tb.ns()); ++i) {
            if (!tb.active(i)) continue;
            bool clamped;
            const double c = species_eval<NC>(tb, i, x, pw, clamped);
            const double cj = clamped ? 0.0 : c;
#pragma unroll
            for (int a = 0; a < NC; ++a) {
                const double sa = tb.s(i, a);
                F[a] = fma(sa, c, F[a]);
                sc[a] = fma(tb.abs_s(i, a), c, sc[a]);
                const double sac = sa * cj;
#pragma unroll
                for (int b = 0; b <= a; ++b) J[a][b] = fma(sac, tb.s(i, b), J[a][b]);
            }
        }
        double rel = 0.0, fn = 0.0, w[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            w[a] = 1.0 / fmax(sc[a], 1e-300);
            const double r = fabs(F[a]) * w[a];
            rel = (r > rel || r != r) ? r : rel;
            fn = fma(r, r, fn);
        }
        if (rel <= tol) { *conv = 1; return it; }
        if (!(rel < 1e300) || stuck) { if (stopped) *stopped = 1; return it; }      // NaN / inf, or stuck
        // fn, fnt: squared weighted residual norms (the Armijo test compares squares)
        // Cholesky of ln10*J (lower triangle), solve L L^T d = -F
        // the diagonal is kept as its reciprocal (rsqrt), so the factorisation
        // and both triangular solves multiply instead of dividing
        double L[NC][NC], Li[NC];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < NC; ++a) {
#pragma unroll
            for (int b = 0; b <= a; ++b) {
                double s = ln10 * J[a][b];
#pragma unroll
                for (int k = 0; k < b; ++k) s -= L[a][k] * L[b][k];
                if (a == b) {
                    if (!(s > 1e-300)) { ok = false; s = 1.0; }
                    Li[a] = rsqrt(s);
                } else {
                    L[a][b] = s * Li[b];
                }
            }
        }
        if (!ok) { if (stopped) *stopped = 1; return it + 1; }
        double d[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            double s = -F[a];
#pragma unroll
            for (int k = 0; k < a; ++k) s -= L[a][k] * d[k];
            d[a] = s * Li[a];
        }
#pragma unroll
        for (int a = NC - 1; a >= 0; --a) {
            double s = d[a];
#pragma unroll
            for (int k = a + 1; k < NC; ++k) s -= L[k][a] * d[k];
            d[a] = s * Li[a];
        }
        // step cap (2 decades), then Armijo backtracking on the weighted residual
        double dmax = 0.0;
#pragma unroll
        for (int a = 0; a < NC; ++a) dmax = fmax(dmax, fabs(d[a]));
        if (dmax > 2.0) {
            const double sfac = 2.0 / dmax;
#pragma unroll
            for (int a = 0; a < NC; ++a) d[a] *= sfac;
        }
        double alpha = 1.0, xt[NC];
        bool accepted = false;
        for (int ls = 0; ls < 40; ++ls) {
#pragma unroll
            for (int a = 0; a < NC; ++a) xt[a] = fmin(fmax(fma(alpha, d[a], x[a]), -30.0), 1.0);
            double Ft[NC];
            eq_residual_t<NC, NS>(tb, T, xt, Ft);
            double fnt = 0.0;
#pragma unroll
            for (int a = 0; a < NC; ++a) { const double r = Ft[a] * w[a]; fnt = fma(r, r, fnt); }
            const double q = 1.0 - 1e-4 * alpha;
            if (fnt < fn * (q * q)) { accepted = true; break; }
            if (alpha < 1e-15) break;
            alpha *= 0.5;
        }
#pragma unroll
        for (int a = 0; a < NC; ++a) x[a] = xt[a];
        // every trial failed: the next iterate is this point to ~1e-12 of a
        // step and fails the same way, so the solve stops after the
        // convergence test at this point
        stuck = !accepted;
    }
    double Fe[NC];
    if (eq_residual_t<NC, NS>(tb, T, x, Fe) <= tol) *conv = 1;
    else if (stuck && stopped) *stopped = 1;
    return max_iter;
}

// The same Newton solve run by a whole warp on one system: every lane holds
// the same iterate and does the same arithmetic, except that the
// backtracking trials of an iteration are spread over the lanes.  Iterates,
// counts and results are those of eq_newton_plain; an iteration that needs
// many trials costs one or two residual evaluations of latency instead of
// up to forty.  For the few slow solves that set the time of the last passes.
template <int NC>
__device__ int eq_newton_warp(const EqDev& e, const double* T, double* x, int max_iter, double tol, int* conv,
                               int* stopped) {
    const double ln10 = 2.302585092994046;
    *conv = 0;
    bool stuck = false;
    for (int it = 0; it < max_iter; ++it) {
        // residual and Jacobian in one pass over the species
        double F[NC], sc[NC], J[NC][NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            F[a] = -T[a]; sc[a] = 0.0;
#pragma unroll
            for (int b = 0; b < NC; ++b) J[a][b] = 0.0;
        }
        Powers<NC> pw;
        pw.set(e, x);
        for (int i = 0; i < e.ns; ++i) {
            if (!e.active[i]) continue;
            bool clamped;
            const double c = species_eval<NC>(e, i, x, pw, clamped);
            const double cj = clamped ? 0.0 : c;
#pragma unroll
            for (int a = 0; a < NC; ++a) {
                const double sa = e.stoich[i][a];
                F[a] = fma(sa, c, F[a]);
                sc[a] = fma(e.absS[i][a], c, sc[a]);
                const double sac = sa * cj;
#pragma unroll
                for (int b = 0; b <= a; ++b) J[a][b] = fma(sac, e.stoich[i][b], J[a][b]);
            }
        }
        double rel = 0.0, fn = 0.0, w[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            w[a] = 1.0 / fmax(sc[a], 1e-300);
            const double r = fabs(F[a]) * w[a];
            rel = (r > rel || r != r) ? r : rel;
            fn = fma(r, r, fn);
        }
        if (rel <= tol) { *conv = 1; return it; }
        if (!(rel < 1e300) || stuck) { if (stopped) *stopped = 1; return it; }      // NaN / inf, or stuck
        // fn, fnt: squared weighted residual norms (the Armijo test compares squares)
        // Cholesky of ln10*J (lower triangle), solve L L^T d = -F
        // the diagonal is kept as its reciprocal (rsqrt), so the factorisation
        // and both triangular solves multiply instead of dividing
        double L[NC][NC], Li[NC];
        bool ok = true;
#pragma unroll
        for (int a = 0; a < NC; ++a) {
#pragma unroll
            for (int b = 0; b <= a; ++b) {
                double s = ln10 * J[a][b];
#pragma unroll
                for (int k = 0; k < b; ++k) s -= L[a][k] * L[b][k];
                if (a == b) {
                    if (!(s > 1e-300)) { ok = false; s = 1.0; }
                    Li[a] = rsqrt(s);
                } else {
                    L[a][b] = s * Li[b];
                }
            }
        }
        if (!ok) { if (stopped) *stopped = 1; return it + 1; }
        double d[NC];
#pragma unroll
        for (int a = 0; a < NC; ++a) {
            double s = -F[a];
#pragma unroll
            for (int k = 0; k < a; ++k) s -= L[a][k] * d[k];
            d[a] = s * Li[a];
        }
#pragma unroll
        for (int a = NC - 1; a >= 0; --a) {
            double s = d[a];
#pragma unroll
            for (int k = a + 1; k < NC; ++k) s -= L[k][a] * d[k];
            d[a] = s * Li[a];
        }
        // step cap (2 decades), then Armijo backtracking on the weighted residual
        double dmax = 0.0;
#pragma unroll
        for (int a = 0; a < NC; ++a) dmax = fmax(dmax, fabs(d[a]));
        if (dmax > 2.0) {
            const double sfac = 2.0 / dmax;
#pragma unroll
            for (int a = 0; a < NC; ++a) d[a] *= sfac;
        }
        // the backtracking trials alpha = 2^-k, k = 0..39, one per lane, 32 at
        // a time; the first k that passes is the one the serial search takes
        const int lane = threadIdx.x & 31;
        double xt[NC];
        bool accepted = false;
        for (int base = 0; base < 40; base += 32) {
            const int kk = base + lane;
            double xk[NC];
#pragma unroll
            for (int a = 0; a < NC; ++a) xk[a] = x[a];
            bool pass = false;
            if (kk < 40) {
                const double alpha = ldexp(1.0, -kk);
#pragma unroll
                for (int a = 0; a < NC; ++a) xk[a] = fmin(fmax(fma(alpha, d[a], x[a]), -30.0), 1.0);
                double Ft[NC];
                eq_residual<NC>(e, T, xk, Ft);
                double fnt = 0.0;
#pragma unroll
                for (int a = 0; a < NC; ++a) { const double r = Ft[a] * w[a]; fnt = fma(r, r, fnt); }
                const double q = 1.0 - 1e-4 * alpha;
                pass = fnt < fn * (q * q);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, pass);
            const int src = bal ? __ffs(bal) - 1 : 39 - base;     // else the last trial (k = 39)
#pragma unroll
            for (int a = 0; a < NC; ++a) xt[a] = __shfl_sync(0xffffffffu, xk[a], src);
            if (bal) { accepted = true; break; }
        }
#pragma unroll
        for (int a = 0; a < NC; ++a) x[a] = xt[a];
        // every trial failed: the next iterate is this point to ~1e-12 of a
        // step and fails the same way, so the solve stops after the
        // convergence test at this point
        stuck = !accepted;
    }
    double Fe[NC];
    if (eq_residual<NC>(e, T, x, Fe) <= tol) *conv = 1;
    else if (stuck && stopped) *stopped = 1;
    return max_iter;
}

// Both variants take the same iterates; above three components the second
// set of residual registers of the reuse variant costs more occupancy than
// the evaluation it saves.
// *stopped (optional) is set when the solve ended before max_iter without
// converging (NaN, singular Jacobian, or every backtracking trial failed):
// continuing from x would repeat the same failure.
// NS > 0: the species count is that compile-time constant (every species
// loop unrolled, so a register array can take the species); 0: e.ns.
template <int NC, int NS = 0>
// cbuf (up to three components): on return it holds the species of x, the
// point the last full evaluation was made at (every return follows one)
__device__ __forceinline__ int eq_newton(const EqDev& e, const double* T, double* x, int max_iter, double tol,
                                         int* conv, int* stopped = nullptr, double* cbuf = nullptr,
                                         int cstride = 0) {
    if constexpr (NC <= 3) return eq_newton_reuse<NC, NS>(TabRun{e}, T, x, max_iter, tol, conv, stopped, cbuf, cstride);
    else return eq_newton_plain<NC, NS>(TabRun{e}, T, x, max_iter, tol, conv, stopped);
}

// the same on a given tableau policy (TabRun or TabFixed)
template <int NC, int NS, class Tab>
__device__ __forceinline__ int eq_newton_t(const Tab& tb, const double* T, double* x, int max_iter, double tol,
                                           int* conv, double* cbuf, int cstride) {
    if constexpr (NC <= 3) return eq_newton_reuse<NC, NS>(tb, T, x, max_iter, tol, conv, nullptr, cbuf, cstride);
    else return eq_newton_plain<NC, NS>(tb, T, x, max_iter, tol, conv, nullptr);
}

// component totals (calc_component_totals, part4_eqsolver.hh:520-538)
template <int NC>
__device__ __forceinline__ void eq_totals(const EqDev& e, const double* species, double* T) {
#pragma unroll
    for (int j = 0; j < NC; ++j) T[j] = 0.0;
    for (int i = 0; i < e.ns; ++i) {
        if (!e.active[i]) continue;
        const double c = fmin(fmax(species[i], 1e-30), 10.0);
#pragma unroll
        for (int j = 0; j < NC; ++j) T[j] = fma(e.stoich[i][j], c, T[j]);
    }
#pragma unroll
    for (int j = 0; j < NC; ++j) T[j] = fmax(T[j], 1e-30);
}

}  // namespace cl
