/*
 * complab_ratelaw.hpp -- the compiled rate-law interface, for host and device.
 *
 * The reference's rate laws are C++ compiled into the program: the user edits
 * defineKinetics.hh (defineRxnKinetics, called by run_kinetics once per voxel,
 * src/complab3d_processors_part1.hh:63-146) and defineAbioticKinetics.hh
 * (defineAbioticRxnKinetics, called by run_abiotic_kinetics, part1.hh:158-249)
 * and rebuilds.  Those functions take std::vector arguments and use lambdas
 * over initializer lists, which device code cannot run.  This header is their
 * replacement: a rate law is a function over fixed-capacity spans (size() and
 * operator[], as the std::vector arguments offer) that compiles for the host
 * with any C++14 compiler and for sm_100a with nvcc, so the same source runs
 * in the transport step on the GPU and, on the host, beside the reference's
 * own header in the tests.
 *
 *   kinetics(B, C, subsR, bioR, mask)   defineRxnKinetics: biomass and
 *                                       concentrations in, rates per second out
 *   abiotic(C, subsR, mask)             defineAbioticRxnKinetics
 *
 * Laws provided: the reference's default network, the Zhao et al. uranium /
 * iron / sulfur model (defineKinetics.hh:223-460 and
 * defineAbioticKinetics.hh:130-218), as zhao::kinetics / zhao::abiotic.  Their
 * constants are the reference's (per-second rate constants, mol/L
 * half-saturations); the code is a restatement over spans.
 */
#ifndef COMPLAB_RATELAW_HPP
#define COMPLAB_RATELAW_HPP

#include <cmath>

#if defined(__CUDACC__)
#define CL_HD __host__ __device__
#else
#define CL_HD
#endif

namespace clrl {

template <class T>
struct span {
    T* p;
    int n;
    CL_HD int size() const { return n; }
    CL_HD T& operator[](int i) const { return p[i]; }
};
typedef span<const double> cspan;
typedef span<double> dspan;

/* std::max / std::min with their exact semantics (the first argument is
 * returned when the comparison is false, so NaN passes through) */
CL_HD inline double vmax(double a, double b) { return (a < b) ? b : a; }
CL_HD inline double vmin(double a, double b) { return (b < a) ? b : a; }
CL_HD inline double monod(double s, double ks) { return s / (ks + s); }
CL_HD inline bool not_finite(double x) {
#if defined(__CUDA_ARCH__)
    return isnan(x) || isinf(x);
#else
    return std::isnan(x) || std::isinf(x);
#endif
}

/* Remove a total consumption `cons` of a dissolved element spread over its
 * buckets I... in proportion to their content: R[i] -= cons * C[i] / tot for
 * every listed bucket present in C (the drawFrom helper of the reference's
 * laws). */
template <int... I>
CL_HD inline void draw_from(double cons, double tot, cspan C, dspan R) {
    if (tot <= 0.0 || cons <= 0.0) return;
    const int idx[sizeof...(I)] = {I...};
    for (unsigned k = 0; k < sizeof...(I); ++k) {
        const int i = idx[k];
        if (i < C.size()) R[i] += -cons * vmax(C[i], 0.0) / tot;
    }
}

/* ---------------------------------------------------------------------------
 * The Zhao network.  Substrate positions: 0 acetate, 1 U(VI), 2 U(IV) (solid),
 * 3 Fe(II), 4-6 Fe(III) easy / medium / hard (solids), 7 sulfate, 8 sulfide,
 * 9 FeS, 10 bicarbonate, 11 H+, 12 methane, 13 S0; 14-23 equilibrium-only
 * components; with the full speciation (more than 24 substrates) positions
 * 24-94 hold the complexes whose aqueous members count toward the dissolved
 * totals.  Biomass pools: 0-3 Geobacter hard / medium / easy / suspended,
 * 4-7 Rhodoferax, 8-9 methanogen attached / suspended, 10-11 sulfate reducer.
 * ------------------------------------------------------------------------- */
namespace zhao {
enum Sub { AC = 0, U6, U4, FE2, FE3E, FE3M, FE3H, SO4, HS, FES, HCO3, HP, CH4, S0 };
enum Pool { GEO_H = 0, GEO_M, GEO_E, GEO_S, RF_H, RF_M, RF_E, RF_S, MT_A, MT_S, SRB_A, SRB_S };
/* U(VI) and its aqueous complexes (the full network's buckets) */
#define CLRL_U6_BUCKETS U6, 65, 66, 67, 68, 69, 70, 71, 72, 73, 74, 75, 76, 77, 78, 79, 80

/* biotic constants (per second, mol/L, mol/mol) */
struct Bio {
    static constexpr double vmax_geo_fe_h = 8.68e-6, vmax_geo_fe_m = 1.74e-5, vmax_geo_fe_e = 1.74e-5;
    static constexpr double vmax_geo_u = 4.05e-6, vmax_rf_fe = 2.08e-6, vmax_mt = 1.62e-4, vmax_srb = 2.55e-5;
    static constexpr double ks_fe = 2.5e-3, ks_u = 2.0e-5, ks_ac_geo = 1.0e-4, ks_fe_rf = 2.5e-4;
    static constexpr double ks_ac_rf = 5.4e-6, ks_ac_mt = 1.0e-5, ks_so4 = 2.0e-4, ks_ac_srb = 7.0e-5;
    static constexpr double ki_fee = 1.0e-3, ki_so4 = 1.6e-3;
    static constexpr double y_geo_fe = 0.035, y_geo_u = 0.012, y_rf = 0.062, y_mt = 0.034, y_srb = 0.041;
    static constexpr double kd = 6.94e-8, kd_geo_e = 2.31e-8;
    static constexpr double k_att = 1.62e-7, k_det_h = 2.08e-7, k_det_m = 2.55e-7, k_det_e = 1.16e-8;
    static constexpr double k_det_rf = 1.62e-7, k_det_mt = 6.94e-8, k_det_srb = 1.62e-7;
    /* per mol acetate */
    static constexpr double fe_per_ac = 4.8, hco3_geo_fe = 1.845, hp_geo_fe = 6.17, hco3_rf_fe = 1.69;
    static constexpr double hp_rf_fe = 6.94, u_per_ac = 3.1, hco3_geo_u = 1.94, hp_geo_u = 8.67;
    static constexpr double so4_per_ac = 0.863, hco3_srb = 1.80, hp_srb = 0.22, ch4_per_ac = 0.93;
    static constexpr double co2_per_ac = 0.93, hp_mt = 0.77;
    static constexpr double eps = 1.0e-12, max_fraction = 0.5, dt = 1.0e-4;
    static constexpr double b_cap = 1.0e-4;      /* attached-biofilm carrying capacity */
};

/* abiotic constants */
struct Abio {
    static constexpr double k_fes = 1.5, k_u_fes = 4.63e-6, k_a4 = 2.41e-4, k_u_hs = 7.16e-3, n_hs = 0.54;
    static constexpr double eps = 1.0e-12, max_fraction = 0.5, dt = 1.0e-4;
    static constexpr double fe3_per_hs = 2.0, hp_r113 = 5.0, u_per_fes = 4.0, hp_r114 = 8.0;
};

/* one pathway's throttle: scale s down so that `draw` takes at most
 * max_fraction of what `avail` holds in one step */
CL_HD inline void cap_scale(double& s, double draw, double avail, double max_fraction, double dt) {
    const double cap = avail * max_fraction / dt;
    if (draw > cap && draw > 0.0) s = vmin(s, cap / draw);
}

/* defineRxnKinetics of the Zhao network (defineKinetics.hh:223-460) */
CL_HD inline void kinetics(cspan B, cspan C, dspan subsR, dspan bioR, int mask) {
    typedef Bio P;
    for (int i = 0; i < subsR.size(); ++i) subsR[i] = 0.0;
    for (int i = 0; i < bioR.size(); ++i) bioR[i] = 0.0;
    if (B.size() < 12 || C.size() < 14) return;
    if (mask < 2) return;

    double ac = vmax(C[AC], 0.0), u6 = vmax(C[U6], 0.0);
    const double fe3e = vmax(C[FE3E], 0.0), fe3m = vmax(C[FE3M], 0.0), fe3h = vmax(C[FE3H], 0.0);
    double so4 = vmax(C[SO4], 0.0);
    const double fes = vmax(C[FES], 0.0);
    if (C.size() > 24) {
        ac += C[56] + C[81] + C[82] + C[83] + C[84] + C[85] + C[86];
        u6 += 2 * (C[65] + C[66] + C[67]) + 3 * (C[68] + C[69] + C[70] + C[71]) + C[72] + C[73] + C[74] + C[75] +
              C[76] + C[77] + C[78] + C[79] + C[80];
        so4 += C[47] + C[48] + C[57];
    }
    const double fe3 = fe3e + fe3m + fe3h;

    double b[12];
    for (int m = 0; m < 12; ++m) b[m] = vmax(B[m], 0.0);

    const double m_geo = monod(ac, P::ks_ac_geo), m_rf = monod(ac, P::ks_ac_rf);
    const double m_mt = monod(ac, P::ks_ac_mt), m_srb = monod(ac, P::ks_ac_srb);
    const double m_u = monod(u6, P::ks_u);
    double free_surface = 1.0 - fes / (fes + fe3 + P::eps);       /* Zhao Eq. 1 */
    free_surface = vmin(vmax(free_surface, 0.0), 1.0);
    const double inhib_mt = (P::ki_fee / (P::ki_fee + fe3e)) * (P::ki_so4 / (P::ki_so4 + so4));

    /* specific acetate-uptake rates of every pathway */
    double geo_fe[3] = {P::vmax_geo_fe_h * b[GEO_H] * monod(fe3h, P::ks_fe) * m_geo,
                        P::vmax_geo_fe_m * b[GEO_M] * monod(fe3m, P::ks_fe) * m_geo,
                        P::vmax_geo_fe_e * b[GEO_E] * monod(fe3e, P::ks_fe) * m_geo};
    double geo_u[4];
    for (int k = 0; k < 4; ++k) geo_u[k] = free_surface * P::vmax_geo_u * b[GEO_H + k] * m_u * m_geo;
    double rf_fe[3] = {P::vmax_rf_fe * b[RF_H] * monod(fe3h, P::ks_fe_rf) * m_rf,
                       P::vmax_rf_fe * b[RF_M] * monod(fe3m, P::ks_fe_rf) * m_rf,
                       P::vmax_rf_fe * b[RF_E] * monod(fe3e, P::ks_fe_rf) * m_rf};
    double mt[2] = {P::vmax_mt * b[MT_A] * m_mt * inhib_mt, P::vmax_mt * b[MT_S] * m_mt * inhib_mt};
    double srb[2] = {P::vmax_srb * b[SRB_A] * monod(so4, P::ks_so4) * m_srb,
                     P::vmax_srb * b[SRB_S] * monod(so4, P::ks_so4) * m_srb};

    /* one common throttle keeps every draw at most half the stock per step */
    double s = 1.0;
    const double ac_draw = geo_fe[0] + geo_fe[1] + geo_fe[2] + geo_u[0] + geo_u[1] + geo_u[2] + geo_u[3] +
                           rf_fe[0] + rf_fe[1] + rf_fe[2] + mt[0] + mt[1] + srb[0] + srb[1];
    cap_scale(s, ac_draw, ac, P::max_fraction, P::dt);
    cap_scale(s, P::fe_per_ac * (geo_fe[0] + rf_fe[0]), fe3h, P::max_fraction, P::dt);
    cap_scale(s, P::fe_per_ac * (geo_fe[1] + rf_fe[1]), fe3m, P::max_fraction, P::dt);
    cap_scale(s, P::fe_per_ac * (geo_fe[2] + rf_fe[2]), fe3e, P::max_fraction, P::dt);
    cap_scale(s, P::u_per_ac * (geo_u[0] + geo_u[1] + geo_u[2] + geo_u[3]), u6, P::max_fraction, P::dt);
    cap_scale(s, P::so4_per_ac * (srb[0] + srb[1]), so4, P::max_fraction, P::dt);
    for (int k = 0; k < 3; ++k) { geo_fe[k] *= s; rf_fe[k] *= s; }
    for (int k = 0; k < 4; ++k) geo_u[k] *= s;
    for (int k = 0; k < 2; ++k) { mt[k] *= s; srb[k] *= s; }

    const double geo_fe_sum = geo_fe[0] + geo_fe[1] + geo_fe[2];
    const double rf_fe_sum = rf_fe[0] + rf_fe[1] + rf_fe[2];
    const double geo_u_sum = geo_u[0] + geo_u[1] + geo_u[2] + geo_u[3];
    const double mt_sum = mt[0] + mt[1], srb_sum = srb[0] + srb[1];

    draw_from<AC, 56, 81, 82, 83, 84, 85, 86>(geo_fe_sum + geo_u_sum + rf_fe_sum + mt_sum + srb_sum, ac, C, subsR);
    subsR[FE3H] = -P::fe_per_ac * (geo_fe[0] + rf_fe[0]);
    subsR[FE3M] = -P::fe_per_ac * (geo_fe[1] + rf_fe[1]);
    subsR[FE3E] = -P::fe_per_ac * (geo_fe[2] + rf_fe[2]);
    subsR[FE2] = +P::fe_per_ac * (geo_fe_sum + rf_fe_sum);
    draw_from<CLRL_U6_BUCKETS>(P::u_per_ac * geo_u_sum, u6, C, subsR);
    subsR[U4] = +P::u_per_ac * geo_u_sum;
    draw_from<SO4, 47, 48, 57>(P::so4_per_ac * srb_sum, so4, C, subsR);
    subsR[HS] = +P::so4_per_ac * srb_sum;
    subsR[CH4] = +P::ch4_per_ac * mt_sum;
    subsR[HCO3] = P::hco3_geo_fe * geo_fe_sum + P::hco3_geo_u * geo_u_sum + P::hco3_rf_fe * rf_fe_sum +
                  P::co2_per_ac * mt_sum + P::hco3_srb * srb_sum;
    subsR[HP] = -P::hp_geo_fe * geo_fe_sum - P::hp_rf_fe * rf_fe_sum - P::hp_srb * srb_sum - P::hp_mt * mt_sum +
                P::hp_geo_u * geo_u_sum;

    /* attachment / detachment between the attached and suspended pools */
    const double geo_att[3] = {P::k_att * b[GEO_S] / 3.0 - P::k_det_h * b[GEO_H],
                               P::k_att * b[GEO_S] / 3.0 - P::k_det_m * b[GEO_M],
                               P::k_att * b[GEO_S] / 3.0 - P::k_det_e * b[GEO_E]};
    const double rf_att[3] = {P::k_att * b[RF_S] / 3.0 - P::k_det_rf * b[RF_H],
                              P::k_att * b[RF_S] / 3.0 - P::k_det_rf * b[RF_M],
                              P::k_att * b[RF_S] / 3.0 - P::k_det_e * b[RF_E]};
    const double mt_att = P::k_att * b[MT_S] - P::k_det_mt * b[MT_A];
    const double srb_att = P::k_att * b[SRB_S] - P::k_det_srb * b[SRB_A];
    /* growth of the attached pools slows to zero at the carrying capacity */
    const double attached = b[GEO_H] + b[GEO_M] + b[GEO_E] + b[RF_H] + b[RF_M] + b[RF_E] + b[MT_A] + b[SRB_A];
    double f_cap = 1.0 - attached / P::b_cap;
    if (f_cap < 0.0) f_cap = 0.0;

    bioR[GEO_H] = f_cap * (P::y_geo_fe * geo_fe[0] + P::y_geo_u * geo_u[0]) - P::kd * b[GEO_H] + geo_att[0];
    bioR[GEO_M] = f_cap * (P::y_geo_fe * geo_fe[1] + P::y_geo_u * geo_u[1]) - P::kd * b[GEO_M] + geo_att[1];
    bioR[GEO_E] = f_cap * (P::y_geo_fe * geo_fe[2] + P::y_geo_u * geo_u[2]) - P::kd_geo_e * b[GEO_E] + geo_att[2];
    bioR[GEO_S] = P::y_geo_u * geo_u[3] - P::kd * b[GEO_S] - (geo_att[0] + geo_att[1] + geo_att[2]);
    bioR[RF_H] = f_cap * (P::y_rf * rf_fe[0]) - P::kd * b[RF_H] + rf_att[0];
    bioR[RF_M] = f_cap * (P::y_rf * rf_fe[1]) - P::kd * b[RF_M] + rf_att[1];
    bioR[RF_E] = f_cap * (P::y_rf * rf_fe[2]) - P::kd * b[RF_E] + rf_att[2];
    bioR[RF_S] = -P::kd * b[RF_S] - (rf_att[0] + rf_att[1] + rf_att[2]);
    bioR[MT_A] = f_cap * (P::y_mt * mt[0]) - P::kd * b[MT_A] + mt_att;
    bioR[MT_S] = P::y_mt * mt[1] - P::kd * b[MT_S] - mt_att;
    bioR[SRB_A] = f_cap * (P::y_srb * srb[0]) - P::kd * b[SRB_A] + srb_att;
    bioR[SRB_S] = P::y_srb * srb[1] - P::kd * b[SRB_S] - srb_att;

    for (int i = 0; i < subsR.size(); ++i) if (not_finite(subsR[i])) subsR[i] = 0.0;
    for (int i = 0; i < bioR.size(); ++i) if (not_finite(bioR[i])) bioR[i] = 0.0;
}

/* defineAbioticRxnKinetics of the Zhao network (defineAbioticKinetics.hh:130-218):
 * R108 U(VI) + sulfide, R112 FeS precipitation, R113 goethite + sulfide,
 * R114 U(VI) on FeS surfaces */
CL_HD inline void abiotic(cspan C, dspan subsR, int mask) {
    typedef Abio P;
    (void)mask;
    for (int i = 0; i < subsR.size(); ++i) subsR[i] = 0.0;
    if (C.size() < 14) return;
    double u6 = vmax(C[U6], 0.0), fe2 = vmax(C[FE2], 0.0);
    const double fe3h = vmax(C[FE3H], 0.0);
    double hs = vmax(C[HS], 0.0);
    const double fes = vmax(C[FES], 0.0);
    if (C.size() > 24) {
        u6 += 2 * (C[65] + C[66] + C[67]) + 3 * (C[68] + C[69] + C[70] + C[71]) + C[72] + C[73] + C[74] + C[75] +
              C[76] + C[77] + C[78] + C[79] + C[80];
        fe2 += C[34] + C[35] + C[36] + C[37] + C[38] + C[39] + C[40] + C[41] + C[83];
        hs += C[43] + C[64];
    }
    const double fe3 = vmax(C[FE3E], 0.0) + vmax(C[FE3M], 0.0) + fe3h;
    double r108 = P::k_u_hs * u6 * std::pow(hs, P::n_hs);
    double r112 = P::k_fes * fe2 * hs;
    double r113 = P::k_a4 * fe3h * hs;
    const double fes_share = fes / (fes + fe3 + P::eps);
    double r114 = P::k_u_fes * fes_share * u6;

    /* per-step limits: no reactant loses more than half its stock */
    const double cap_fe2 = fe2 * P::max_fraction / P::dt;
    if (r112 > cap_fe2) r112 = cap_fe2;
    const double cap_feh = fe3h * P::max_fraction / P::dt;
    if (P::fe3_per_hs * r113 > cap_feh && r113 > 0.0) r113 = cap_feh / P::fe3_per_hs;
    const double hs_draw = r108 + r112 + r113;
    const double cap_hs = hs * P::max_fraction / P::dt;
    if (hs_draw > cap_hs && hs_draw > 0.0) { const double s = cap_hs / hs_draw; r108 *= s; r112 *= s; r113 *= s; }
    const double u_draw = r108 + r114;
    const double cap_u = u6 * P::max_fraction / P::dt;
    if (u_draw > cap_u && u_draw > 0.0) { const double s = cap_u / u_draw; r108 *= s; r114 *= s; }
    const double cap_fes = fes * P::max_fraction / P::dt;
    if (r114 / P::u_per_fes > cap_fes && r114 > 0.0) r114 = cap_fes * P::u_per_fes;

    draw_from<CLRL_U6_BUCKETS>(r108 + r114, u6, C, subsR);
    subsR[U4] = +r108 + r114;
    subsR[FE3H] = -P::fe3_per_hs * r113;
    draw_from<FE2, 34, 35, 36, 37, 38, 39, 40, 41, 83>(r112, fe2, C, subsR);
    subsR[FE2] += P::fe3_per_hs * r113 + r114 / P::u_per_fes;
    subsR[FES] = +r112 - r114 / P::u_per_fes;
    draw_from<HS, 43, 64>(r108 + r112 + r113, hs, C, subsR);
    subsR[SO4] = +r114 / P::u_per_fes;
    subsR[S0] = +r108 + r113;
    subsR[HP] = +r108 + r112 - P::hp_r113 * r113 - (P::hp_r114 / P::u_per_fes) * r114;
    for (int i = 0; i < subsR.size(); ++i) if (not_finite(subsR[i])) subsR[i] = 0.0;
}
#undef CLRL_U6_BUCKETS
}  // namespace zhao

}  // namespace clrl

#endif /* COMPLAB_RATELAW_HPP */
