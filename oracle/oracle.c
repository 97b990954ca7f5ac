/*
 * oracle.c -- FP64 CPU oracle (test infrastructure only; see oracle.h).
 *
 * Every function restates one reference processor or one Palabos algorithm
 * the reference calls; the citation sits above each.  Parity with Palabos
 * itself is unpinned (Palabos v2.3.0 is not vendored with the reference).
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define THRD 1e-12                 /* src/complab3d_processors.hh: thrd */

/* sizeof(cl_config) as this library was compiled, for binding checks */
int orc_config_size(void) { return (int)sizeof(cl_config); }
#define COMPLAB_THRD 1e-14         /* src/complab_functions.hh:64 */

/* ---------------------------------------------------------------- lattices */
/* D3Q19 in Palabos order: the first nine have a negative leading component,
 * opp(i) = i +/- 9. */
static const int C19[19][3] = {
    {0,0,0},
    {-1,0,0},{0,-1,0},{0,0,-1},{-1,-1,0},{-1,1,0},{-1,0,-1},{-1,0,1},{0,-1,-1},{0,-1,1},
    {1,0,0},{0,1,0},{0,0,1},{1,1,0},{1,-1,0},{1,0,1},{1,0,-1},{0,1,1},{0,1,-1}};
static const double T19[19] = {
    1.0/3,
    1.0/18,1.0/18,1.0/18,1.0/36,1.0/36,1.0/36,1.0/36,1.0/36,1.0/36,
    1.0/18,1.0/18,1.0/18,1.0/36,1.0/36,1.0/36,1.0/36,1.0/36,1.0/36};
static int opp19(int i) { return i == 0 ? 0 : (i <= 9 ? i + 9 : i - 9); }

/* D3Q7 (Palabos AdvectionDiffusionD3Q7Descriptor): t0 = 1/4, ti = 1/8, cs2 = 1/4.
 * The reference's increment code adds dC/4 to g[0] and dC/8 to the others
 * (src/complab3d_processors_part1.hh:108), consistent with these weights. */
static const int C7[7][3] = {{0,0,0},{-1,0,0},{0,-1,0},{0,0,-1},{1,0,0},{0,1,0},{0,0,1}};
static const double T7[7] = {0.25,0.125,0.125,0.125,0.125,0.125,0.125};
static int opp7(int i) { return i == 0 ? 0 : (i <= 3 ? i + 3 : i - 3); }

static inline int64_t site(const cl_config* c, int x, int y, int z) {
    return ((int64_t)x * c->ny + y) * c->nz + z;
}
static inline int wrap(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

static int in_list(int v, const int32_t* list, int n) {
    for (int i = 0; i < n; ++i) if (list[i] == v) return 1;
    return 0;
}

/* Dynamics assignment of NSdomainSetup (src/complab_functions.hh:245-294) and
 * soluteDomainSetup (:296-340): default BGK everywhere, then pore codes, then
 * bounce_back, then solid (NoDynamics), then biofilm codes, later wins. */
void orc_classes_from_mask(const cl_config* cfg, const uint8_t* mask,
                           uint8_t* ns_class, uint8_t* ade_class) {
    int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    for (int64_t n = 0; n < N; ++n) {
        int m = mask[n];
        uint8_t ns = ORC_FLUID, ad = ORC_FLUID;
        if (in_list(m, cfg->pore_codes, cfg->n_pore_codes)) { ns = ORC_FLUID; ad = ORC_FLUID; }
        if (cfg->bb_code > 0 && m == cfg->bb_code) { ns = ORC_BB; ad = ORC_BB; }
        if (cfg->solid_code >= 0 && m == cfg->solid_code) { ns = ORC_NODYN; ad = ORC_NODYN; }
        if (in_list(m, cfg->bio_codes, cfg->n_bio_codes)) {
            ns = (cfg->perm_ratio > COMPLAB_THRD) ? ORC_BIO : ORC_BB;
            ad = ORC_BIO;
        }
        ns_class[n] = ns; ade_class[n] = ad;
    }
}

/* ------------------------------------------------------------------- flow */
/* Palabos bgk_ma2_equilibrium with invRho = 1 (IncBGKdynamics): deviation form */
static inline double feq_inc(int i, double rhoBar, const double j[3], double jSqr) {
    double cj = C19[i][0]*j[0] + C19[i][1]*j[1] + C19[i][2]*j[2];
    return T19[i] * (rhoBar + 3.0*cj + 4.5*cj*cj - 1.5*jSqr);
}

static double omega_ns(const cl_config* cfg, int cls) {
    double om = 1.0 / cfg->tau_ns;
    if (cls == ORC_BIO) om = 1.0 / (cfg->perm_ratio * (1.0/om - 0.5) + 0.5);  /* complab_functions.hh:271 */
    return om;
}

/* PressureGradient (src/complab_functions.hh:72-84) generalised to given end
 * densities: rho(x) linear from rho_in at x=0 to rho_out at x=nx-1; u = 0.
 * Non-BGK cells hold their dynamics' zero equilibrium (fbar = 0). */
void orc_flow_init(const cl_config* cfg, const uint8_t* ns_class, double* f) {
    int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    for (int x = 0; x < cfg->nx; ++x)
        for (int y = 0; y < cfg->ny; ++y)
            for (int z = 0; z < cfg->nz; ++z) {
                int64_t n = site(cfg, x, y, z);
                double rho = cfg->rho_in + (cfg->rho_out - cfg->rho_in) * (double)x / (double)(cfg->nx - 1);
                int bgk = ns_class[n] == ORC_FLUID || ns_class[n] == ORC_BIO;
                for (int i = 0; i < 19; ++i) f[i*N + n] = bgk ? T19[i] * (rho - 1.0) : 0.0;
            }
}

/* Regularized density boundary (Latt et al. 2008), as Palabos
 * RegularizedDensityBoundaryDynamics over IncBGK: the normal momentum from the
 * known populations, tangential momentum zero, PiNeq from the known
 * populations with bounce-back of the non-equilibrium part, populations rebuilt
 * as feq + t_i/(2 cs^4) Q_i:PiNeq.  side = -1 west (x=0), +1 east (x=nx-1). */
static void regularize_pressure(double* fb, double rhoBar, int side, double j[3]) {
    double s0 = 0, sn = 0;
    for (int i = 0; i < 19; ++i) {
        if (C19[i][0] == 0) s0 += fb[i];
        else if (C19[i][0] == side) sn += fb[i];          /* known: leaving through this face */
    }
    /* west: j_x = rhoBar - s0 - 2*s_minus ; east: j_x = s0 + 2*s_plus - rhoBar */
    j[0] = (side < 0) ? (rhoBar - s0 - 2.0*sn) : (s0 + 2.0*sn - rhoBar);
    j[1] = 0.0; j[2] = 0.0;
    double jSqr = j[0]*j[0];
    double pi[6] = {0,0,0,0,0,0};   /* xx yy zz xy xz yz */
    for (int i = 0; i < 19; ++i) {
        double w;
        if (C19[i][0] == 0) w = 1.0;
        else if (C19[i][0] == side) w = 2.0;
        else continue;
        double fneq = fb[i] - feq_inc(i, rhoBar, j, jSqr);
        const int* c = C19[i];
        pi[0] += w*c[0]*c[0]*fneq; pi[1] += w*c[1]*c[1]*fneq; pi[2] += w*c[2]*c[2]*fneq;
        pi[3] += w*c[0]*c[1]*fneq; pi[4] += w*c[0]*c[2]*fneq; pi[5] += w*c[1]*c[2]*fneq;
    }
    for (int i = 0; i < 19; ++i) {
        const int* c = C19[i];
        const double cs2 = 1.0/3.0;
        double qpi = (c[0]*c[0]-cs2)*pi[0] + (c[1]*c[1]-cs2)*pi[1] + (c[2]*c[2]-cs2)*pi[2]
                   + 2.0*(c[0]*c[1]*pi[3] + c[0]*c[2]*pi[4] + c[1]*c[2]*pi[5]);
        fb[i] = feq_inc(i, rhoBar, j, jSqr) + T19[i] * 4.5 * qpi;
    }
}

/* One collideAndStream.  Collide per class (IncBGK, BounceBack swap, NoDynamics
 * identity), then push streaming; y,z periodic; a population leaving through an
 * x face is reflected into its own site's opposite slot (what Palabos's
 * swap-based streaming leaves in a slot with no upstream neighbour). */
double orc_flow_step(const cl_config* cfg, const uint8_t* ns_class,
                     const double* f_in, double* f_out) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    const int64_t N = (int64_t)nx * ny * nz;
    double esum = 0.0; int64_t ecount = 0;
    #pragma omp parallel for collapse(2) reduction(+:esum,ecount) schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int64_t n = site(cfg, x, y, z);
                double fb[19], fo[19];
                for (int i = 0; i < 19; ++i) fb[i] = f_in[i*N + n];
                int cls = ns_class[n];
                if (cls == ORC_NODYN) {
                    for (int i = 0; i < 19; ++i) fo[i] = fb[i];
                } else if (cls == ORC_BB) {
                    for (int i = 0; i < 19; ++i) fo[i] = fb[opp19(i)];
                } else {
                    double om = omega_ns(cfg, cls);
                    double rhoBar = 0, j[3] = {0,0,0};
                    if (x == 0 || x == nx - 1) {
                        rhoBar = (x == 0 ? cfg->rho_in : cfg->rho_out) - 1.0;
                        regularize_pressure(fb, rhoBar, x == 0 ? -1 : 1, j);
                    } else {
                        for (int i = 0; i < 19; ++i) {
                            rhoBar += fb[i];
                            j[0] += C19[i][0]*fb[i]; j[1] += C19[i][1]*fb[i]; j[2] += C19[i][2]*fb[i];
                        }
                    }
                    double jSqr = j[0]*j[0] + j[1]*j[1] + j[2]*j[2];
                    for (int i = 0; i < 19; ++i)
                        fo[i] = fb[i]*(1.0 - om) + om*feq_inc(i, rhoBar, j, jSqr);
                    esum += 0.5*jSqr; ecount += 1;
                }
                for (int i = 0; i < 19; ++i) {
                    int xd = x + C19[i][0];
                    if (xd < 0 || xd >= nx) { f_out[opp19(i)*N + n] = fo[i]; continue; }
                    int yd = wrap(y + C19[i][1], ny), zd = wrap(z + C19[i][2], nz);
                    f_out[i*N + site(cfg, xd, yd, zd)] = fo[i];
                }
            }
    return ecount ? esum / (double)ecount : 0.0;
}

/* util::ValueTracer(u=1, L=1000, eps) of Palabos: window deltaT = L/u/2 = 500
 * values; converged when the window is full and stddev/average < eps (sample
 * stddev, n-1); a NaN ratio counts as "diverged" and also stops the loop.
 * Loop shape of src/complab.cpp:607-611. */
int orc_flow_solve(const cl_config* cfg, const uint8_t* ns_class, double* f,
                   double* f_tmp, int max_it, double eps, double* energy_hist) {
    const int W = 500;
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    double* win = (double*)malloc(sizeof(double) * W);
    int count = 0, head = 0, it = 0, diverged = 0;
    for (it = 0; it < max_it; ++it) {
        double e = orc_flow_step(cfg, ns_class, f, f_tmp);
        memcpy(f, f_tmp, sizeof(double) * 19 * N);
        if (energy_hist) energy_hist[it] = e;
        win[head] = e; head = (head + 1) % W; if (count < W) ++count;
        if (count >= W) {
            double avg = 0; for (int k = 0; k < W; ++k) avg += win[k];
            avg /= W;
            double sq = 0; for (int k = 0; k < W; ++k) sq += (win[k]-avg)*(win[k]-avg);
            double ratio = sqrt(sq / (W - 1)) / avg;
            if (isnan(ratio)) { diverged = 1; break; }
            if (ratio < eps) break;
        }
    }
    free(win);
    return diverged ? -1 : it;
}

/* computeDensity / computeVelocity per site.  BGK cells: rho = 1 + sum fbar,
 * u = j (IncBGK: velocity is j).  Pressure-boundary cells: the prescribed rho
 * and the boundary's j.  BounceBack / NoDynamics: rho as stored, u = 0. */
void orc_flow_macro(const cl_config* cfg, const uint8_t* ns_class, const double* f,
                    double* rho, double* u) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    const int64_t N = (int64_t)nx * ny * nz;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int64_t n = site(cfg, x, y, z);
                double fb[19], rb = 0, j[3] = {0,0,0};
                for (int i = 0; i < 19; ++i) fb[i] = f[i*N + n];
                int cls = ns_class[n];
                if ((cls == ORC_FLUID || cls == ORC_BIO) && (x == 0 || x == nx - 1)) {
                    rb = (x == 0 ? cfg->rho_in : cfg->rho_out) - 1.0;
                    double tmp[19]; memcpy(tmp, fb, sizeof tmp);
                    regularize_pressure(tmp, rb, x == 0 ? -1 : 1, j);
                } else {
                    for (int i = 0; i < 19; ++i) {
                        rb += fb[i];
                        j[0] += C19[i][0]*fb[i]; j[1] += C19[i][1]*fb[i]; j[2] += C19[i][2]*fb[i];
                    }
                    if (!(cls == ORC_FLUID || cls == ORC_BIO)) { j[0] = j[1] = j[2] = 0; }
                }
                if (rho) rho[n] = 1.0 + rb;
                if (u) { u[n] = j[0]; u[N + n] = j[1]; u[2*N + n] = j[2]; }
            }
}

/* -------------------------------------------------------------- transport */
static int is_reactive(const cl_config* cfg, int x, int m) {
    return x > 0 && x < cfg->nx - 1 && m != cfg->solid_code && m != cfg->bb_code;
}

/* initializeAtEquilibrium(c0, u=0) of every solute lattice
 * (src/complab_functions.hh:334-336); the prescribed boundary densities are
 * the Dirichlet values, or for a zero-gradient face the density next to it
 * (FlatAdiabaticBoundaryFunctional3D run by lattice.initialize()). */
void orc_ade_init(const cl_config* cfg, orc_state* st) {
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    const int64_t P = (int64_t)cfg->ny * cfg->nz;
    for (int s = 0; s < cfg->n_solutes; ++s) {
        if (cfg->immobile[s]) {
            for (int64_t n = 0; n < N; ++n) st->imm[s*N + n] = cfg->c0[s];
        } else {
            for (int i = 0; i < 7; ++i)
                for (int64_t n = 0; n < N; ++n) st->g[(s*7 + i)*N + n] = T7[i] * cfg->c0[s];
        }
        for (int64_t p = 0; p < P; ++p) {
            st->rho_bc[(s*2 + 0)*P + p] = cfg->left_type[s] == CL_BC_DIRICHLET ? cfg->left_value[s] : cfg->c0[s];
            st->rho_bc[(s*2 + 1)*P + p] = cfg->right_type[s] == CL_BC_DIRICHLET ? cfg->right_value[s] : cfg->c0[s];
        }
    }
    /* initPhaseLattice3D (dissolutionVOP.hh:195-229): grain phases take their
     * id where the geometry holds their material; then each grain phase with
     * initial_fill > 0 seeds that inventory there (initializeScalarLattice3D,
     * complab.cpp:858-871) */
    if (cfg->dissol_enabled && st->phase) {
        for (int64_t n = 0; n < N; ++n) {
            uint8_t pid = 0;
            for (int k = 0; k < cfg->n_phases; ++k) {
                if (cfg->phases[k].is_precipitate) continue;
                if (cfg->phases[k].material == st->mask[n]) { pid = (uint8_t)cfg->phases[k].id; break; }
            }
            st->phase[n] = pid;
        }
        for (int k = 0; k < cfg->n_phases; ++k) {
            const cl_phase* ph = &cfg->phases[k];
            if (ph->is_precipitate || !(ph->initial_fill > 0.0)) continue;
            const int s = ph->substrate;
            for (int64_t n = 0; n < N; ++n) {
                if (st->mask[n] != ph->material) continue;
                if (cfg->immobile[s]) st->imm[s*N + n] = ph->initial_fill;
                else for (int i = 0; i < 7; ++i) st->g[(s*7 + i)*N + n] = T7[i] * ph->initial_fill;
            }
        }
    }
}

/* computeDensity of every site.  A dynamic cell on an x face answers with its
 * prescribed density (the boundary dynamics stores it: the Dirichlet value, or
 * for a zero-gradient face the value FlatAdiabaticBoundaryFunctional3D copied
 * from the neighbour plane after the last stream). */
void orc_solute_density(const cl_config* cfg, const orc_state* st, int s, double* out) {
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz, P = (int64_t)cfg->ny * cfg->nz;
    if (cfg->immobile[s]) { memcpy(out, st->imm + s*N, sizeof(double)*N); return; }
    for (int64_t n = 0; n < N; ++n) {
        double r = 0; for (int i = 0; i < 7; ++i) r += st->g[(s*7 + i)*N + n];
        out[n] = r;
    }
    for (int side = 0; side < 2; ++side) {
        int64_t base = side == 0 ? 0 : N - P;
        for (int64_t p = 0; p < P; ++p) {
            int cls = st->ade_class[base + p];
            if (cls == ORC_FLUID || cls == ORC_BIO) out[base + p] = st->rho_bc[(s*2 + side)*P + p];
        }
    }
}

/* Table-driven rate law (defineRxnKinetics / defineAbioticRxnKinetics ABI:
 * defineKinetics.hh:223-229, defineAbioticKinetics.hh:130).  abiotic selects
 * the reactions with microbe < 0, biotic those with microbe >= 0 plus decay. */
void orc_rates(const cl_config* cfg, int abiotic, const double* C, const double* B,
               double* subsR, double* bioR) {
    for (int s = 0; s < cfg->n_solutes; ++s) subsR[s] = 0.0;
    if (bioR) for (int m = 0; m < cfg->n_microbes; ++m) bioR[m] = 0.0;
    for (int k = 0; k < cfg->n_rxn; ++k) {
        const cl_rxn* r = &cfg->rxn[k];
        if ((r->microbe < 0) != (abiotic != 0)) continue;
        double rate = r->k;
        if (r->microbe >= 0) {
            double b = B[r->microbe];
            if (!(b > 0.0)) continue;
            rate *= b;
        }
        for (int j = 0; j < r->n_monod; ++j) {
            double c = C[r->monod_s[j]]; if (c < 0) c = 0;
            rate *= c / (r->monod_ks[j] + c);
        }
        if (r->ksp > 0.0) {
            /* saturation-index drive (an extension; the reference has no
             * solubility products): max(P / ksp - 1, 0) */
            double prod = 1.0;
            for (int j = 0; j < r->n_mass; ++j) {
                double c = C[r->mass_s[j]]; if (c < 0) c = 0;
                prod *= c;
            }
            rate *= fmax(prod / r->ksp - 1.0, 0.0);
        } else {
            for (int j = 0; j < r->n_mass; ++j) {
                double c = C[r->mass_s[j]]; if (c < 0) c = 0;
                rate *= c;
            }
        }
        for (int s = 0; s < cfg->n_solutes; ++s) subsR[s] += r->nu[s] * rate;
        if (r->microbe >= 0 && bioR) bioR[r->microbe] += r->yield * rate;
    }
    if (!abiotic && bioR)
        for (int m = 0; m < cfg->n_microbes; ++m) {
            double b = B[m] > 0 ? B[m] : 0.0;
            bioR[m] -= cfg->decay[m] * b;
        }
    for (int s = 0; s < cfg->n_solutes; ++s) if (!isfinite(subsR[s])) subsR[s] = 0.0;
    if (bioR) for (int m = 0; m < cfg->n_microbes; ++m) if (!isfinite(bioR[m])) bioR[m] = 0.0;
}

/* Surrogate reaction type at one voxel (run_surrogate3D,
 * src/complab3d_processors_surrogate.hh:94-295, with MetabolicConfig's
 * conversions, complab3d_metabolic.hh:481-519).  C: densities before
 * update_rxnLattices; B: floored biomass.  Adds thresholded increments to
 * D (solutes) and DB (biomass). */
static void orc_surrogate_voxel(const cl_config* cfg, const cl_surrogate_net* nets, const double* C,
                                const double* B, double* D, double* DB) {
    const int S = cfg->n_solutes;
    double conc[CL_MAX_SOLUTES], draw[CL_MAX_SOLUTES];
    int any = 0;
    for (int o = 0; o < cfg->n_srg; ++o) if (B[cfg->srg[o].microbe] > THRD) any = 1;
    if (!any) return;
    for (int s = 0; s < S; ++s) { conc[s] = C[s] > THRD ? C[s] : 0.0; draw[s] = 0.0; }
    for (int o = 0; o < cfg->n_srg; ++o) {
        const cl_srg_organism* g = &cfg->srg[o];
        const cl_surrogate_net* net = &nets[g->net];
        const double b = B[g->microbe];
        if (!(b > THRD)) continue;
        double fin[CL_MAX_SOLUTES], fout[CL_MAX_SOLUTES];
        const double denom = b * g->mw * cfg->dt;
        for (int s = 0; s < S; ++s) {
            const double av = conc[s];
            const double mm = (g->kc[s] + av > 0.0) ? av / (g->kc[s] + av) : 0.0;
            double exh = 0.0;                                  /* exhaustionFlux */
            if (denom > 1e-30) { exh = -av * 3.6e6 / denom; if (exh < -1e4) exh = -1e4; }
            double v = g->vmax[s] > THRD ? g->vmax[s] * mm : -exh * mm;
            const double cap = -exh;
            if (cap > 0.0 && v > cap) v = cap;
            fin[s] = v; fout[s] = v;
        }
        double xin[CL_SRG_MAX_WIDTH], y[CL_SRG_MAX_WIDTH];
        for (int i = 0; i < net->widths[0]; ++i) {
            int kind = g->in_kind[i], idx = g->in_index[i];
            xin[i] = kind == CL_SRG_IN_FIN ? fin[idx] : kind == CL_SRG_IN_CONC ? conc[idx] : b;
        }
        orc_surrogate_forward(net, xin, y, 1);
        double mu = 0.0;
        for (int q = 0; q < net->widths[net->n_layers]; ++q) {
            if (g->out_kind[q] == CL_SRG_OUT_GROWTH) mu = y[q];
            else fout[g->out_index[q]] = y[q];
        }
        if (mu < 1e-8 || !isfinite(mu)) mu = 0.0;
        double dB = (fabs(mu) < THRD) ? -g->kd * b * cfg->dt : mu * b * cfg->dt / 3600.0;
        if (dB + b < 0.0) dB = -b;
        if (fabs(dB) > THRD) DB[g->microbe] += dB;
        for (int s = 0; s < S; ++s) draw[s] += -fout[s] * b * g->mw * cfg->dt / 3.6e6;
    }
    for (int s = 0; s < S; ++s) {
        double d = draw[s];
        if (fabs(d) <= THRD) continue;
        if (d + conc[s] < 0.0) d = -conc[s];
        if (d > 0.0) d = 0.0;
        if (fabs(d) > THRD) D[s] += d;
    }
}

/* Speciation --------------------------------------------------------------- */
#define MIN_CONC 1e-30
#define MAX_CONC 10.0
#define MIN_LOG_C (-30.0)
#define MAX_LOG_C 1.0

static int eq_species_active(const cl_eq_system* sys, int i) {
    for (int j = 0; j < sys->n_comp; ++j) if (fabs(sys->stoich[i][j]) > 1e-10) return 1;
    return 0;
}

/* calc_species (part4_eqsolver.hh:442-496) for equilibrium species */
void orc_eq_species(const cl_eq_system* sys, const double* x, double* c) {
    for (int i = 0; i < sys->n_species; ++i) {
        if (!eq_species_active(sys, i)) { c[i] = 0.0; continue; }
        double lc = sys->logk[i];
        for (int j = 0; j < sys->n_comp; ++j) lc += sys->stoich[i][j] * x[j];
        if (lc > MAX_LOG_C) lc = MAX_LOG_C;
        if (lc < MIN_LOG_C) lc = MIN_LOG_C;
        c[i] = pow(10.0, lc);
    }
}

/* calc_component_totals (part4_eqsolver.hh:520-538) */
void orc_eq_totals(const cl_eq_system* sys, const double* species, double* totals) {
    for (int j = 0; j < sys->n_comp; ++j) {
        double t = 0.0;
        for (int i = 0; i < sys->n_species; ++i) {
            if (!eq_species_active(sys, i)) continue;
            double c = species[i];
            if (c > MAX_CONC) c = MAX_CONC;
            if (c < MIN_CONC) c = MIN_CONC;
            t += sys->stoich[i][j] * c;
        }
        totals[j] = t > MIN_CONC ? t : MIN_CONC;
    }
}

/* initial guess of solve_equilibrium_anderson (part4_eqsolver.hh:977-994),
 * identical in the Newton reserve (NR_reserve.hh:527-540) */
void orc_eq_cold_start(const cl_eq_system* sys, const double* species, double* x0) {
    for (int j = 0; j < sys->n_comp; ++j) {
        double c = 1e-7;
        int idx = sys->comp_species[j];
        if (idx >= 0 && idx < sys->n_species) c = species[idx];
        if (c > MAX_CONC) c = MAX_CONC;
        if (c < MIN_CONC) c = MIN_CONC;
        x0[j] = log10(c);
    }
}

/* relative mass-balance residual max_j |sum_i S_ij c_i - T_j| / sum_i |S_ij| c_i */
static double eq_eval(const cl_eq_system* sys, const double* T, const double* x,
                      double* F, double* c) {
    orc_eq_species(sys, x, c);
    double rel = 0.0;
    for (int j = 0; j < sys->n_comp; ++j) {
        double f = -T[j], sc = 0.0;
        for (int i = 0; i < sys->n_species; ++i) {
            f += sys->stoich[i][j] * c[i];
            sc += fabs(sys->stoich[i][j]) * c[i];
        }
        F[j] = f;
        double r = fabs(f) / (sc > 1e-300 ? sc : 1e-300);
        if (!(r <= rel)) rel = r;   /* NaN-propagating max */
    }
    return rel;
}

double orc_eq_residual(const cl_eq_system* sys, const double* totals, const double* x) {
    double F[CL_MAX_COMP], c[CL_MAX_SPECIES];
    return eq_eval(sys, totals, x, F, c);
}

/* Newton-Raphson in log10 free components, restating solve_equilibrium_NR
 * (src/complab3d_processors_part4_eqsolver_NR_reserve.hh:512-615): residual
 * F = S^T c - T (:309-328), Jacobian J = ln10 S^T diag(c) S (:356-377),
 * Gaussian elimination with partial pivoting (:414-481), Armijo backtracking
 * with alpha halving, at most 40 trials (:577-598).  Four documented
 * deviations make it converge on the 5x14 random tableaux, where the reserve
 * as written stalls on 83% of cold starts (its line search on the unweighted
 * ||F||_2 accepts only vanishing steps when totals span decades):
 *   - stopping test: relative mass-balance residual <= tol (reserve: absolute
 *     ||F||_2 < 1e-12);
 *   - species held at a clamp bound contribute nothing to J (the derivative of
 *     the clamped value), so J matches F;
 *   - the Newton step is scaled so that no component moves more than 2 decades;
 *   - the Armijo merit is ||F_j / sum_i |S_ij| c_i||_2 with the weights of the
 *     current iterate.
 * A solve whose 40 backtracking trials all fail stops at once (the reserve
 * would repeat the same failing iteration at a point moved by ~1e-12 of a
 * step until max_iter). */
int orc_eq_newton(const cl_eq_system* sys, const double* totals, double* x,
                  int max_iter, double tol, int* converged) {
    const int nc = sys->n_comp, ns = sys->n_species;
    double F[CL_MAX_COMP], c[CL_MAX_SPECIES], Ft[CL_MAX_COMP], ct[CL_MAX_SPECIES];
    double xt[CL_MAX_COMP];
    *converged = 0;
    if (nc == 0) { *converged = 1; return 0; }
    for (int it = 0; it < max_iter; ++it) {
        double rel = eq_eval(sys, totals, x, F, c);
        if (rel <= tol) { *converged = 1; return it; }
        if (!isfinite(rel)) return it;
        /* J = ln10 * S^T diag(c) S ; A = [J | -F] */
        double A[CL_MAX_COMP][CL_MAX_COMP + 1], cj[CL_MAX_SPECIES], w[CL_MAX_COMP];
        const double ln10 = 2.302585092994046;
        for (int i = 0; i < ns; ++i) {
            double lc = sys->logk[i];
            for (int j = 0; j < nc; ++j) lc += sys->stoich[i][j] * x[j];
            cj[i] = (lc > MAX_LOG_C || lc < MIN_LOG_C) ? 0.0 : c[i];
        }
        for (int a = 0; a < nc; ++a) {
            for (int b = 0; b < nc; ++b) {
                double s = 0;
                for (int i = 0; i < ns; ++i) s += sys->stoich[i][a] * sys->stoich[i][b] * cj[i];
                A[a][b] = ln10 * s;
            }
            A[a][nc] = -F[a];
            double sc = 0;
            for (int i = 0; i < ns; ++i) sc += fabs(sys->stoich[i][a]) * c[i];
            w[a] = 1.0 / (sc > 1e-300 ? sc : 1e-300);
        }
        int ok = 1;
        for (int k = 0; k < nc; ++k) {
            int p = k; double mx = fabs(A[k][k]);
            for (int r = k + 1; r < nc; ++r) if (fabs(A[r][k]) > mx) { mx = fabs(A[r][k]); p = r; }
            if (!(mx > 1e-300)) { ok = 0; break; }
            if (p != k) for (int q = 0; q <= nc; ++q) { double t = A[k][q]; A[k][q] = A[p][q]; A[p][q] = t; }
            for (int r = k + 1; r < nc; ++r) {
                double fct = A[r][k] / A[k][k];
                for (int q = k; q <= nc; ++q) A[r][q] -= fct * A[k][q];
            }
        }
        if (!ok) return it + 1;
        double d[CL_MAX_COMP];
        for (int k = nc - 1; k >= 0; --k) {
            double s = A[k][nc];
            for (int q = k + 1; q < nc; ++q) s -= A[k][q] * d[q];
            d[k] = s / A[k][k];
        }
        double dmax = 0; for (int j = 0; j < nc; ++j) if (fabs(d[j]) > dmax) dmax = fabs(d[j]);
        if (dmax > 2.0) for (int j = 0; j < nc; ++j) d[j] *= 2.0 / dmax;
        double fn = 0; for (int j = 0; j < nc; ++j) fn += (F[j]*w[j])*(F[j]*w[j]);
        fn = sqrt(fn);
        double alpha = 1.0;
        int accepted = 0;
        for (int ls = 0; ls < 40; ++ls) {
            for (int j = 0; j < nc; ++j) {
                double v = x[j] + alpha * d[j];
                if (v > MAX_LOG_C) v = MAX_LOG_C;
                if (v < MIN_LOG_C) v = MIN_LOG_C;
                xt[j] = v;
            }
            eq_eval(sys, totals, xt, Ft, ct);
            double fnt = 0; for (int j = 0; j < nc; ++j) fnt += (Ft[j]*w[j])*(Ft[j]*w[j]);
            fnt = sqrt(fnt);
            if (fnt < fn * (1.0 - 1e-4 * alpha)) { accepted = 1; break; }
            if (alpha < 1e-15) break;
            alpha *= 0.5;
        }
        for (int j = 0; j < nc; ++j) x[j] = xt[j];
        /* no trial down to 2^-39 of the step decreased the merit: the next
         * iterate is the same point to ~1e-12 and fails the same way, so the
         * solve stops here (not converged unless this point already is) */
        if (!accepted) {
            double F2[CL_MAX_COMP], c2[CL_MAX_SPECIES];
            if (eq_eval(sys, totals, x, F2, c2) <= tol) *converged = 1;
            return it + 1;
        }
    }
    double F2[CL_MAX_COMP], c2[CL_MAX_SPECIES];
    if (eq_eval(sys, totals, x, F2, c2) <= tol) *converged = 1;
    return max_iter;
}

/* ---- the reference's live solver: PCF + Anderson acceleration -------------
 * Restates EquilibriumChemistry<T>::calculate_species_concentrations
 * (src/complab3d_processors_part4_eqsolver.hh:1187-1214) and what it calls:
 * calc_component_totals (:520-538), calc_species (:442-496),
 * calc_reactive_product_sums (:540-640), pcf_residual (:664-726),
 * qr_decomposition (:817-868), solve_upper_triangular (:887-904) and
 * solve_equilibrium_anderson (:952-1172), with the reference's constants
 * (condition limit 1e10, mixing 1).  The arithmetic is done in the
 * reference's order (plain double multiply and add, glibc pow / log10), so
 * built with the same compiler flags it reproduces the reference's iterates. */
#define PCF_COND_TOL 1e10
#define PCF_MAX_DEPTH 16
/* std::min / std::max as the reference calls them: a NaN first argument
 * passes through */
static inline double smin(double a, double b) { return (b < a) ? b : a; }
static inline double smax(double a, double b) { return (a < b) ? b : a; }

/* calc_species: equilibrium species from the log free components; the others
 * keep their input value (clamped), as does a species whose power overflows */
static void pcf_species(const cl_eq_system* sys, const double* x, const double* init, double* c) {
    for (int i = 0; i < sys->n_species; ++i) {
        if (!eq_species_active(sys, i)) { c[i] = init[i] > MIN_CONC ? smin(init[i], MAX_CONC) : MIN_CONC; continue; }
        double lc = sys->logk[i];
        for (int j = 0; j < sys->n_comp; ++j) lc += sys->stoich[i][j] * x[j];
        lc = smax(smin(lc, MAX_LOG_C), MIN_LOG_C);
        double v = pow(10.0, lc);
        if (isnan(v) || isinf(v)) v = init[i] > MIN_CONC ? init[i] : MIN_CONC;
        c[i] = smax(smin(v, MAX_CONC), MIN_CONC);
    }
}

/* the smallest positive stoichiometric coefficient of each component (at most 1) */
static double pcf_mu_min(const cl_eq_system* sys, int j) {
    double mu_min = 1.0;
    for (int i = 0; i < sys->n_species; ++i) {
        if (!eq_species_active(sys, i)) continue;
        const double mu = sys->stoich[i][j];
        if (mu > 1e-10 && mu < mu_min) mu_min = mu;
    }
    return mu_min;
}

/* pcf_residual: f_j = log10(S_P / S_R) / mu_min_j, clamped to +-10; 0 for a
 * non-finite value and for an absent component (T_j <= 1e-18) */
static void pcf_correction(const cl_eq_system* sys, const double* T, const double* x, const double* init,
                           double* f) {
    double c[CL_MAX_SPECIES];
    pcf_species(sys, x, init, c);
    for (int j = 0; j < sys->n_comp; ++j) {
        double pos = 0.0, neg = 0.0;
        for (int i = 0; i < sys->n_species; ++i) {
            if (!eq_species_active(sys, i)) continue;
            const double mu = sys->stoich[i][j];
            const double ci = smax(c[i], MIN_CONC);
            if (mu > 1e-15) pos += mu * ci;
            else if (mu < -1e-15) neg += fabs(mu) * ci;
        }
        double sr, sp;
        if (T[j] >= 0.0) { sr = pos; sp = T[j] + neg; }
        else { sr = fabs(T[j]) + pos; sp = neg; }
        sr = smax(sr, MIN_CONC);
        sp = smax(sp, MIN_CONC);
        double v = (1.0 / pcf_mu_min(sys, j)) * (log10(sp) - log10(sr));
        v = smax(smin(v, 10.0), -10.0);
        if (isnan(v) || isinf(v)) v = 0.0;
        if (T[j] <= 1e-18) v = 0.0;
        f[j] = v;
    }
}

static double pcf_norm(const double* v, int n) {
    double s = 0.0;
    for (int k = 0; k < n; ++k) s += v[k] * v[k];
    return sqrt(s);
}

/* classical Gram-Schmidt on the columns cols[0..m-1] (length n); R upper
 * triangle; *cond = max / min of the |R_jj| above 1e-30 */
static void pcf_qr(double cols[][CL_MAX_COMP], int m, int n, double Q[][CL_MAX_COMP],
                   double R[][PCF_MAX_DEPTH], double* cond) {
    double rmax = 0.0, rmin = DBL_MAX;
    for (int j = 0; j < m; ++j) {
        for (int k = 0; k < n; ++k) Q[j][k] = cols[j][k];
        for (int i = 0; i < j; ++i) {
            double d = 0.0;
            for (int k = 0; k < n; ++k) d += Q[i][k] * cols[j][k];
            R[i][j] = d;
            for (int k = 0; k < n; ++k) Q[j][k] -= R[i][j] * Q[i][k];
        }
        R[j][j] = pcf_norm(Q[j], n);
        if (R[j][j] > 1e-15)
            for (int k = 0; k < n; ++k) Q[j][k] /= R[j][j];
        const double a = fabs(R[j][j]);
        if (a > rmax) rmax = a;
        if (a > 1e-30 && a < rmin) rmin = a;
    }
    *cond = m == 0 ? 1.0 : (rmin > 1e-30 ? rmax / rmin : DBL_MAX);
}

/* one solve; species_in as given to calculate_species_concentrations.  Returns
 * 1 if ||f||_2 < tol was reached; *iters = getLastIterations() */
int orc_pcf_solve(const cl_eq_system* sys, const double* species_in, double* species_out, int* iters) {
    const int nc = sys->n_comp, ns = sys->n_species;
    const int depth = sys->anderson_depth > 0 ? (sys->anderson_depth < PCF_MAX_DEPTH - 1 ? sys->anderson_depth
                                                                                         : PCF_MAX_DEPTH - 2) : 4;
    double T[CL_MAX_COMP], x[CL_MAX_COMP], xn[CL_MAX_COMP], f[CL_MAX_COMP];
    *iters = 0;
    if (nc == 0 || ns == 0) {
        for (int i = 0; i < ns; ++i) species_out[i] = species_in[i];
        return 1;
    }
    orc_eq_totals(sys, species_in, T);
    orc_eq_cold_start(sys, species_in, x);
    /* history of iterates and corrections, oldest first; depth + 2 entries at most */
    double hx[PCF_MAX_DEPTH][CL_MAX_COMP], hf[PCF_MAX_DEPTH][CL_MAX_COMP];
    int hn = 0;
    pcf_correction(sys, T, x, species_in, f);
    for (int j = 0; j < nc; ++j) xn[j] = smax(smin(x[j] + f[j], MAX_LOG_C), MIN_LOG_C);
    for (int j = 0; j < nc; ++j) { hx[0][j] = x[j]; hf[0][j] = f[j]; x[j] = xn[j]; }
    hn = 1;
    int conv = 0;
    for (int it = 1; it < sys->max_iter; ++it) {
        *iters = it;
        pcf_correction(sys, T, x, species_in, f);
        if (pcf_norm(f, nc) < sys->tol) { conv = 1; break; }
        for (int j = 0; j < nc; ++j) { hx[hn][j] = x[j]; hf[hn][j] = f[j]; }
        ++hn;
        int m = hn - 1 < depth ? hn - 1 : depth;
        if (m < 1) {
            for (int j = 0; j < nc; ++j) xn[j] = x[j] + f[j];
        } else {
            double dF[PCF_MAX_DEPTH][CL_MAX_COMP], dX[PCF_MAX_DEPTH][CL_MAX_COMP];
            double Q[PCF_MAX_DEPTH][CL_MAX_COMP], R[PCF_MAX_DEPTH][PCF_MAX_DEPTH], cond;
            for (int i = 0; i < m; ++i) {
                const int a = hn - m - 1 + i;
                for (int j = 0; j < nc; ++j) { dF[i][j] = hf[a + 1][j] - hf[a][j]; dX[i][j] = hx[a + 1][j] - hx[a][j]; }
            }
            int first = 0;      /* columns dropped from the front */
            pcf_qr(dF, m, nc, Q, R, &cond);
            while (cond > PCF_COND_TOL && m - first > 1) {
                ++first;
                pcf_qr(dF + first, m - first, nc, Q, R, &cond);
            }
            const int mm = m - first;
            double g[PCF_MAX_DEPTH], qf[PCF_MAX_DEPTH];
            for (int i = 0; i < mm; ++i) {
                double d = 0.0;
                for (int k = 0; k < nc; ++k) d += Q[i][k] * f[k];
                qf[i] = d;
            }
            for (int i = mm - 1; i >= 0; --i) {
                double v = qf[i];
                for (int k = i + 1; k < mm; ++k) v -= R[i][k] * g[k];
                if (fabs(R[i][i]) > 1e-30) v /= R[i][i];
                g[i] = v;
            }
            double sx[CL_MAX_COMP] = {0}, sf[CL_MAX_COMP] = {0};
            for (int i = 0; i < mm; ++i)
                for (int j = 0; j < nc; ++j) {
                    sx[j] += dX[first + i][j] * g[i];
                    sf[j] += dF[first + i][j] * g[i];
                }
            for (int j = 0; j < nc; ++j) xn[j] = x[j] - sx[j] + 1.0 * (f[j] - sf[j]);
        }
        for (int j = 0; j < nc; ++j) {
            double v = smax(smin(xn[j], MAX_LOG_C), MIN_LOG_C);
            if (isnan(v) || isinf(v)) v = x[j];
            x[j] = v;
        }
        /* keep the depth + 1 newest entries */
        while (hn > depth + 1) {
            for (int a = 1; a < hn; ++a)
                for (int j = 0; j < nc; ++j) { hx[a - 1][j] = hx[a][j]; hf[a - 1][j] = hf[a][j]; }
            --hn;
        }
    }
    pcf_species(sys, x, species_in, species_out);
    for (int i = 0; i < ns; ++i) {
        double v = species_out[i];
        if (isnan(v) || isinf(v)) v = species_in[i] > MIN_CONC ? smin(species_in[i], MAX_CONC) : MIN_CONC;
        species_out[i] = smax(smin(v, MAX_CONC), MIN_CONC);
    }
    return conv;
}

void orc_pcf_batch(const cl_eq_system* sys, const double* species_in, double* species_out, int32_t* iters,
                   uint8_t* conv, int64_t n) {
    const int ns = sys->n_species;
    #pragma omp parallel for schedule(dynamic, 64)
    for (int64_t k = 0; k < n; ++k) {
        int it = 0;
        const int cv = orc_pcf_solve(sys, species_in + k*ns, species_out + k*ns, &it);
        if (iters) iters[k] = it;
        if (conv) conv[k] = (uint8_t)cv;
    }
}

void orc_eq_batch(const cl_eq_system* sys, const double* totals, const double* cold_species,
                  double* x_io, int32_t* iters, uint8_t* status, int64_t n, int start) {
    const int nc = sys->n_comp, ns = sys->n_species;
    #pragma omp parallel for schedule(dynamic, 256)
    for (int64_t k = 0; k < n; ++k) {
        double x[CL_MAX_COMP];
        if (start == CL_EQ_START_COLD) orc_eq_cold_start(sys, cold_species + k*ns, x);
        else for (int j = 0; j < nc; ++j) x[j] = x_io[k*nc + j];
        int conv = 0;
        int limit = (start == CL_EQ_START_COLD) ? sys->max_iter : sys->warm_iter;
        int it = orc_eq_newton(sys, totals + k*nc, x, limit, sys->tol, &conv);
        uint8_t stt = 0;
        if (!conv && start != CL_EQ_START_COLD) {
            orc_eq_cold_start(sys, cold_species + k*ns, x);
            it += orc_eq_newton(sys, totals + k*nc, x, sys->max_iter, sys->tol, &conv);
            stt = 1;
        }
        if (!conv) stt = 2;
        for (int j = 0; j < nc; ++j) x_io[k*nc + j] = x[j];
        if (iters) iters[k] = it;
        if (status) status[k] = stt;
    }
}

/* ---- per-voxel reaction processors (shared by both pass structures) ---- */
typedef struct {
    const cl_config* cfg;
    orc_state* st;
    int64_t N;
    int any_bio, any_srg, any_abio;
} rx_ctx;

static double vox_dens(const rx_ctx* r, int s, int64_t n) {
    const int64_t N = r->N;
    if (r->cfg->immobile[s]) return r->st->imm[s*N + n];
    const double* g = r->st->g;
    return g[(s*7+0)*N+n] + g[(s*7+1)*N+n] + g[(s*7+2)*N+n] + g[(s*7+3)*N+n] +
           g[(s*7+4)*N+n] + g[(s*7+5)*N+n] + g[(s*7+6)*N+n];
}

/* g_i += t_i * d (the reference's g[0] += d/4, g[1..6] += d/8) */
static void vox_apply(const rx_ctx* r, int s, int64_t n, double d) {
    const int64_t N = r->N;
    if (r->cfg->immobile[s]) { r->st->imm[s*N + n] += d; return; }
    for (int i = 0; i < 7; ++i) r->st->g[(s*7 + i)*N + n] += T7[i] * d;
}

/* run_kinetics (part1.hh:63-146) and run_surrogate3D deposit into the same
 * dC/dB lattices, each contribution only above thrd; update_rxnLattices
 * (:338-429) applies the sums above thrd */
static void vox_kinetics(const rx_ctx* r, int64_t n) {
    const cl_config* cfg = r->cfg;
    const int S = cfg->n_solutes, M = cfg->n_microbes;
    const int64_t N = r->N;
    double C[CL_MAX_SOLUTES], Bm[CL_MAX_MICROBES], R[CL_MAX_SOLUTES], BR[CL_MAX_MICROBES];
    double dC[CL_MAX_SOLUTES], dB[CL_MAX_MICROBES];
    for (int s = 0; s < S; ++s) { double c = vox_dens(r, s, n); C[s] = c < THRD ? 0.0 : c; dC[s] = 0.0; }
    /* a microbe solved by LBM (microbe_carrier): its biomass is the density
     * of its carrier solute, its dB goes to that lattice */
    for (int b = 0; b < M; ++b) {
        const int cr = cfg->microbe_carrier[b] - 1;
        double v = cr >= 0 ? C[cr] : r->st->bio[b*N + n];
        Bm[b] = v < THRD ? 0.0 : v; dB[b] = 0.0;
    }
    if (r->any_bio) {
        if (r->st->kin) r->st->kin(Bm, M, C, S, R, BR, r->st->mask[n]);
        else orc_rates(cfg, 0, C, Bm, R, BR);
        for (int s = 0; s < S; ++s) {
            double d = R[s] * cfg->dt;
            dC[s] = (d > THRD || d < -THRD) ? d : 0.0;
        }
        for (int b = 0; b < M; ++b) {
            double d = BR[b] * cfg->dt;
            dB[b] = (d > THRD || d < -THRD) ? d : 0.0;
        }
    }
    if (r->any_srg) orc_surrogate_voxel(cfg, r->st->srg_nets, C, Bm, dC, dB);
    for (int b = 0; b < M; ++b)
        if (cfg->microbe_carrier[b] > 0) { dC[cfg->microbe_carrier[b] - 1] += dB[b]; dB[b] = 0.0; }
    for (int s = 0; s < S; ++s) if (dC[s] > THRD || dC[s] < -THRD) vox_apply(r, s, n, dC[s]);
    for (int b = 0; b < M; ++b) if (dB[b] > THRD || dB[b] < -THRD) r->st->bio[b*N + n] += dB[b];
}

/* run_abiotic_kinetics (part1.hh:158-249) or surfaceAbioticKinetics3D
 * (precipitationVOP.hh:53-145): the thresholded increments of one voxel
 * (zero where the surface gate does not fire) */
static void vox_abiotic(const rx_ctx* r, int x, int y, int z, int64_t n, double* dC) {
    const cl_config* cfg = r->cfg;
    const orc_state* st = r->st;
    const int S = cfg->n_solutes;
    for (int s = 0; s < S; ++s) dC[s] = 0.0;
    int fire = 1;
    if (cfg->precip_enabled && cfg->abiotic_surface_only) {
        static const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
        fire = 0;
        for (int d = 0; d < 6 && !fire; ++d) {
            int xa = x + d6[d][0];
            if (xa < 0 || xa > cfg->nx - 1) continue;
            int nb = st->mask[site(cfg, xa, wrap(y + d6[d][1], cfg->ny), wrap(z + d6[d][2], cfg->nz))];
            if (nb == cfg->solid_code || nb == cfg->bb_code) fire = 1;
        }
    }
    if (!fire) return;
    double C[CL_MAX_SOLUTES], R[CL_MAX_SOLUTES];
    for (int s = 0; s < S; ++s) { double c = vox_dens(r, s, n); C[s] = c < THRD ? 0.0 : c; }
    if (st->abio) st->abio(C, S, R, st->mask[n]);
    else orc_rates(cfg, 1, C, NULL, R, NULL);
    for (int s = 0; s < S; ++s) {
        double d = R[s] * cfg->dt;
        dC[s] = (d > THRD || d < -THRD) ? d : 0.0;
    }
}

/* SolidPhase by id (DissolutionConfig::byId, dissolutionVOP.hh:176-180) */
static const cl_phase* phase_by_id(const cl_config* cfg, int pid) {
    for (int k = 0; k < cfg->n_phases; ++k) if (cfg->phases[k].id == pid) return &cfg->phases[k];
    return NULL;
}

/* surfaceDissolutionKinetics3D (dissolutionVOP.hh:265-435) at one voxel:
 * water = mean solute density over the open face neighbours (x in 1..nx-2,
 * y/z inside the domain, not solid or bounce-back), the phase's rate law,
 * at most half the mineral per step, the mineral decrement into the voxel's
 * own dC and the products split evenly into the open neighbours' dC. */
static void vox_dissolve(const rx_ctx* r, int x, int y, int z, double* dab) {
    const cl_config* cfg = r->cfg;
    const orc_state* st = r->st;
    const int S = cfg->n_solutes, nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    const int64_t N = r->N, n = site(cfg, x, y, z);
    const int pid = st->phase[n];
    if (pid <= 0) return;
    const cl_phase* ph = phase_by_id(cfg, pid);
    if (!ph || ph->substrate < 0 || ph->substrate >= S) return;
    const int sM = ph->substrate;
    const double mineral = vox_dens(r, sM, n);
    if (!(mineral > THRD)) return;
    static const int d6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};
    int64_t open[6];
    int nOpen = 0;
    for (int d = 0; d < 6; ++d) {
        int ax = x + d6[d][0], ay = y + d6[d][1], az = z + d6[d][2];
        if (ax < 1 || ax > nx - 2 || ay < 0 || ay > ny - 1 || az < 0 || az > nz - 1) continue;
        int64_t q = site(cfg, ax, ay, az);
        int m = st->mask[q];
        if (m == cfg->solid_code || m == cfg->bb_code) continue;
        open[nOpen++] = q;
    }
    if (nOpen == 0 && cfg->dissol_surface_only) return;
    double water[CL_MAX_SOLUTES];
    for (int s = 0; s < S; ++s) water[s] = 0.0;
    if (nOpen > 0) {
        for (int k = 0; k < nOpen; ++k)
            for (int s = 0; s < S; ++s) water[s] += vox_dens(r, s, open[k]);
        for (int s = 0; s < S; ++s) water[s] /= (double)nOpen;
    }
    for (int s = 0; s < S; ++s) if (water[s] < 0.0) water[s] = 0.0;
    /* defineDissolutionRate as a table: rate = k * mineral * prod water[mass_s] */
    double rate = ph->k * (mineral > 0.0 ? mineral : 0.0);
    for (int j = 0; j < ph->n_mass; ++j) rate *= water[ph->mass_s[j]];
    double mineralR = -rate, subsR[CL_MAX_SOLUTES];
    for (int s = 0; s < S; ++s) subsR[s] = ph->nu[s] * rate;
    if (isnan(mineralR) || isinf(mineralR)) mineralR = 0.0;
    for (int s = 0; s < S; ++s) if (isnan(subsR[s]) || isinf(subsR[s])) subsR[s] = 0.0;
    if (!(mineralR < 0.0)) return;
    double dM = mineralR * cfg->dt;
    double scale = 1.0;
    const double maxRemove = 0.5 * mineral;
    if (-dM > maxRemove) scale = maxRemove / (-dM);
    dM *= scale;
    if (!(-dM > THRD)) return;
    dab[sM*N + n] += dM;
    if (nOpen > 0) {
        for (int s = 0; s < S; ++s) {
            if (s == sM) continue;
            const double released = subsR[s] * cfg->dt * scale;
            if (fabs(released) <= THRD) continue;
            const double perFace = released / (double)nOpen;
            for (int k = 0; k < nOpen; ++k) dab[s*N + open[k]] += perFace;
        }
    }
}

/* run_equilibrium_biotic (part4_eqsolver.hh:1355-1494) with the Newton solve
 * or the reference's PCF + Anderson; returns 1 if it did not converge */
static int vox_equilibrium(const rx_ctx* r, int64_t n) {
    const cl_config* cfg = r->cfg;
    const int S = cfg->n_solutes;
    const cl_eq_system* sys = &cfg->eq;
    double conc[CL_MAX_SPECIES], T[CL_MAX_COMP], xx[CL_MAX_COMP], eqc[CL_MAX_SPECIES];
    for (int s = 0; s < S; ++s) { double c = vox_dens(r, s, n); conc[s] = c > MIN_CONC ? c : MIN_CONC; }
    if (sys->solver == CL_EQ_SOLVER_PCF) {
        /* the reference's live solver: its result is applied whether or not it converged */
        int it = 0;
        const int cv = orc_pcf_solve(sys, conc, eqc, &it);
        if (r->st->eq_iters) r->st->eq_iters[n] = it;
        for (int s = 0; s < S && s < sys->n_species; ++s) {
            double d = eqc[s] - conc[s];
            double mx = 0.1 * fabs(conc[s]); if (mx < 1e-9) mx = 1e-9;
            if (fabs(d) > mx) d = d > 0 ? mx : -mx;
            if (conc[s] + d < 1e-20) d = 1e-20 - conc[s];
            if (fabs(d) > THRD) vox_apply(r, s, n, d);
        }
        return cv ? 0 : 1;
    }
    orc_eq_totals(sys, conc, T);
    orc_eq_cold_start(sys, conc, xx);
    int conv = 0;
    int it = orc_eq_newton(sys, T, xx, sys->max_iter, sys->tol, &conv);
    if (r->st->eq_iters) r->st->eq_iters[n] = it;
    if (!conv) return 1;
    orc_eq_species(sys, xx, eqc);
    for (int s = 0; s < S && s < sys->n_species; ++s) {
        double e = eq_species_active(sys, s) ? eqc[s]
                 : (conc[s] > MIN_CONC ? (conc[s] < MAX_CONC ? conc[s] : MAX_CONC) : MIN_CONC);
        if (e > MAX_CONC) e = MAX_CONC;
        if (e < MIN_CONC) e = MIN_CONC;
        double d = e - conc[s];
        double mx = 0.1 * fabs(conc[s]); if (mx < 1e-9) mx = 1e-9;
        if (fabs(d) > mx) d = d > 0 ? mx : -mx;
        if (conc[s] + d < 1e-20) d = 1e-20 - conc[s];
        if (fabs(d) > THRD) vox_apply(r, s, n, d);
    }
    return 0;
}

/* The reaction stage of a transport step, between collide and stream
 * (src/complab.cpp:1264-1374): run_kinetics -> update_rxnLattices -> dC reset
 * -> run_abiotic_kinetics | surfaceAbioticKinetics3D (+ surfaceDissolutionKinetics3D)
 * -> update_abiotic_rxnLattices -> run_equilibrium_biotic.  Returns the
 * number of Newton solves that did not converge. */
int64_t orc_reaction_stage(const cl_config* cfg, orc_state* st) {
    return orc_reaction_ops(cfg, st, ORC_OP_ALL);
}

/* the processors of the reaction stage selected by ops (ORC_OP_*), each as
 * in orc_reaction_stage; kinetics and surrogate share one increment lattice */
int64_t orc_reaction_ops(const cl_config* cfg, orc_state* st, int ops) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, S = cfg->n_solutes, M = cfg->n_microbes;
    const int64_t N = (int64_t)nx * ny * nz;
    int64_t nonconv = 0;
    int n_bio = 0, n_abio = 0;
    for (int k = 0; k < cfg->n_rxn; ++k) { if (cfg->rxn[k].microbe >= 0) ++n_bio; else ++n_abio; }
    rx_ctx rc;
    rc.cfg = cfg; rc.st = st; rc.N = N;
    rc.any_bio = cfg->enable_kinetics && (n_bio > 0 || M > 0) && (ops & ORC_OP_KINETICS);
    rc.any_srg = cfg->n_srg > 0 && st->srg_nets && (ops & ORC_OP_SURROGATE);
    rc.any_abio = cfg->enable_abiotic && S > 0 && (n_abio > 0 || st->abio != NULL) && (ops & ORC_OP_ABIOTIC);
    const int dissol = cfg->dissol_enabled && cfg->n_phases > 0 && st->phase && (ops & ORC_OP_ABIOTIC);
    const int eq = cfg->use_equilibrium && (ops & ORC_OP_EQUILIBRIUM);
    if (!dissol) {
        /* processors run over the whole lattice in turn, and each reads only
         * its own voxel, so one pass per voxel is exact */
        #pragma omp parallel for collapse(2) reduction(+:nonconv) schedule(dynamic, 4)
        for (int x = 1; x < nx - 1; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    int64_t n = site(cfg, x, y, z);
                    if (!is_reactive(cfg, x, st->mask[n])) continue;
                    double dC[CL_MAX_SOLUTES];
                    if (rc.any_bio || rc.any_srg) vox_kinetics(&rc, n);
                    if (rc.any_abio) {
                        vox_abiotic(&rc, x, y, z, n, dC);
                        for (int s = 0; s < S; ++s) if (dC[s] > THRD || dC[s] < -THRD) vox_apply(&rc, s, n, dC[s]);
                    }
                    if (eq) nonconv += vox_equilibrium(&rc, n);
                }
    } else {
        /* surfaceDissolutionKinetics3D writes the dC of face neighbours, so the
         * processors run as separate whole-lattice passes, as the reference does */
        #pragma omp parallel for collapse(2) schedule(dynamic, 4)
        for (int x = 1; x < nx - 1; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    int64_t n = site(cfg, x, y, z);
                    if (!is_reactive(cfg, x, st->mask[n])) continue;
                    if (rc.any_bio || rc.any_srg) vox_kinetics(&rc, n);
                }
        /* dC = dC0 (complab.cpp:1328 / :1359) */
        double* dab = (double*)calloc((size_t)S * N, sizeof(double));
        if (rc.any_abio) {
            #pragma omp parallel for collapse(2) schedule(dynamic, 4)
            for (int x = 1; x < nx - 1; ++x)
                for (int y = 0; y < ny; ++y)
                    for (int z = 0; z < nz; ++z) {
                        int64_t n = site(cfg, x, y, z);
                        if (!is_reactive(cfg, x, st->mask[n])) continue;
                        double dC[CL_MAX_SOLUTES];
                        vox_abiotic(&rc, x, y, z, n, dC);
                        for (int s = 0; s < S; ++s) dab[s*N + n] = dC[s];
                    }
        }
        /* the scatter into neighbours runs serially in the reference's voxel order */
        for (int x = 1; x < nx - 1; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) vox_dissolve(&rc, x, y, z, dab);
        /* update_abiotic_rxnLattices (part1.hh:258-336): interior x, not solid or
         * bounce-back; with dissol_apply_at_walls the walls' mineral decrement too */
        #pragma omp parallel for collapse(2) schedule(static)
        for (int x = 1; x < nx - 1; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    int64_t n = site(cfg, x, y, z);
                    if (!is_reactive(cfg, x, st->mask[n]) && !cfg->dissol_apply_at_walls) continue;
                    for (int s = 0; s < S; ++s) {
                        double d = dab[s*N + n];
                        if (d > THRD || d < -THRD) vox_apply(&rc, s, n, d);
                    }
                }
        free(dab);
        if (eq) {
            #pragma omp parallel for collapse(2) reduction(+:nonconv) schedule(dynamic, 4)
            for (int x = 1; x < nx - 1; ++x)
                for (int y = 0; y < ny; ++y)
                    for (int z = 0; z < nz; ++z) {
                        int64_t n = site(cfg, x, y, z);
                        if (!is_reactive(cfg, x, st->mask[n])) continue;
                        nonconv += vox_equilibrium(&rc, n);
                    }
        }
    }

    return nonconv;
}

/* One transport step in the order of src/complab.cpp:1252-1374,1849-1857:
 *   collide (mobile solutes; boundary cells complete their unknown population
 *   from the prescribed density first) -> run_kinetics -> update_rxnLattices ->
 *   dC reset -> run_abiotic_kinetics | surfaceAbioticKinetics3D ->
 *   update_abiotic_rxnLattices -> run_equilibrium_biotic -> stream ->
 *   FlatAdiabaticBoundaryFunctional3D on zero-gradient faces. */
int64_t orc_transport_step(const cl_config* cfg, orc_state* st) {
    orc_collide(cfg, st);
    const int64_t nonconv = orc_reaction_stage(cfg, st);
    orc_stream(cfg, st);
    return nonconv;
}

/* collide of every mobile solute in place (the first part of a step) */
void orc_collide(const cl_config* cfg, orc_state* st) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, S = cfg->n_solutes;
    const int64_t N = (int64_t)nx * ny * nz, P = (int64_t)ny * nz;
    double* g = st->g;

    /* ---- collide (AdvectionDiffusionBGKdynamics, BounceBack, NoDynamics) ---- */
    #pragma omp parallel for collapse(2) schedule(static)
    for (int x = 0; x < nx; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                int64_t n = site(cfg, x, y, z);
                int cls = st->ade_class[n];
                for (int s = 0; s < S; ++s) {
                    if (cfg->immobile[s]) continue;
                    double gi[7];
                    for (int i = 0; i < 7; ++i) gi[i] = g[(s*7 + i)*N + n];
                    if (cls == ORC_NODYN) continue;
                    if (cls == ORC_BB) {
                        for (int i = 0; i < 7; ++i) g[(s*7 + i)*N + n] = gi[opp7(i)];
                        continue;
                    }
                    if (x == 0 || x == nx - 1) {
                        /* AdvectionDiffusionBoundaryDynamics: the one unknown population
                         * (entering through the face) = prescribed rho - sum of the others */
                        int unk = (x == 0) ? 4 : 1;
                        double rb = st->rho_bc[(s*2 + (x == 0 ? 0 : 1))*P + (int64_t)y*nz + z];
                        double sum = 0; for (int i = 0; i < 7; ++i) if (i != unk) sum += gi[i];
                        gi[unk] = rb - sum;
                    }
                    double om = (cls == ORC_BIO) ? cfg->omega_bio[s] : cfg->omega_pore[s];
                    double rho = 0; for (int i = 0; i < 7; ++i) rho += gi[i];
                    double ux = st->u[n], uy = st->u[N + n], uz = st->u[2*N + n];
                    for (int i = 0; i < 7; ++i) {
                        double cu = C7[i][0]*ux + C7[i][1]*uy + C7[i][2]*uz;
                        double geq = T7[i] * rho * (1.0 + 4.0*cu);
                        g[(s*7 + i)*N + n] = gi[i] - om*(gi[i] - geq);
                    }
                }
            }

}

/* stream every mobile solute (push, periodic y/z, reflect at x faces), then
 * the zero-gradient faces (the last part of a step) */
void orc_stream(const cl_config* cfg, orc_state* st) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, S = cfg->n_solutes;
    const int64_t N = (int64_t)nx * ny * nz, P = (int64_t)ny * nz;
    double* g = st->g;
    /* ---- stream (push, periodic y/z, reflect at x faces) ---- */
    for (int s = 0; s < S; ++s) {
        if (cfg->immobile[s]) continue;
        double* gs = g + (int64_t)s*7*N;
        double* go = st->g_tmp + (int64_t)s*7*N;
        #pragma omp parallel for collapse(2) schedule(static)
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    int64_t n = site(cfg, x, y, z);
                    for (int i = 0; i < 7; ++i) {
                        int xd = x + C7[i][0];
                        if (xd < 0 || xd >= nx) { go[opp7(i)*N + n] = gs[i*N + n]; continue; }
                        go[i*N + site(cfg, xd, wrap(y + C7[i][1], ny), wrap(z + C7[i][2], nz))] = gs[i*N + n];
                    }
                }
        memcpy(gs, go, sizeof(double) * 7 * N);
        /* FlatAdiabaticBoundaryFunctional3D<0,-1/+1>: boundary density := neighbour's */
        for (int side = 0; side < 2; ++side) {
            int bt = side == 0 ? cfg->left_type[s] : cfg->right_type[s];
            if (bt != CL_BC_NEUMANN) continue;
            int xn = side == 0 ? 1 : nx - 2;
            for (int y = 0; y < ny; ++y)
                for (int z = 0; z < nz; ++z) {
                    int64_t n = site(cfg, xn, y, z);
                    double r = 0; for (int i = 0; i < 7; ++i) r += gs[i*N + n];
                    st->rho_bc[(s*2 + side)*P + (int64_t)y*nz + z] = r;
                }
        }
    }
}

/* precipNodeConversion3D (src/precipitationVOP.hh:158-219) */
int64_t orc_precip_convert(const cl_config* cfg, orc_state* st) {
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    int64_t changed = 0;
    int s = cfg->precip_substrate;
    for (int64_t n = 0; n < N; ++n) {
        int m = st->mask[n];
        if (m == cfg->solid_code || m == cfg->bb_code) continue;
        double p = cfg->immobile[s] ? st->imm[s*N + n] : 0.0;
        if (!cfg->immobile[s]) for (int i = 0; i < 7; ++i) p += st->g[(s*7 + i)*N + n];
        if (p >= cfg->max_precip_rho) {
            if (m != cfg->precip_code) ++changed;
            st->mask[n] = (uint8_t)cfg->precip_code;
            /* stamp the precipitate phase so dissolution can find the voxel */
            if (cfg->precip_phase_id > 0 && st->phase) st->phase[n] = (uint8_t)cfg->precip_phase_id;
        }
    }
    return changed;
}

/* dissolNodeConversion3D (src/dissolutionVOP.hh:459-527): a phase voxel whose
 * mineral fell below reopen_fraction * full_density becomes the first pore
 * code (2 when none is declared) and loses its phase id. */
int64_t orc_dissol_convert(const cl_config* cfg, orc_state* st) {
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    const int pore = cfg->n_pore_codes > 0 ? cfg->pore_codes[0] : 2;
    int64_t changed = 0;
    if (!st->phase) return 0;
    for (int64_t n = 0; n < N; ++n) {
        const int pid = st->phase[n];
        if (pid <= 0) continue;
        const cl_phase* ph = phase_by_id(cfg, pid);
        if (!ph || ph->substrate < 0 || ph->substrate >= cfg->n_solutes) continue;
        if (!(ph->full_density > 0.0)) continue;
        const int s = ph->substrate;
        double mineral = cfg->immobile[s] ? st->imm[s*N + n] : 0.0;
        if (!cfg->immobile[s]) for (int i = 0; i < 7; ++i) mineral += st->g[(s*7 + i)*N + n];
        if (mineral < cfg->reopen_fraction * ph->full_density) {
            if (st->mask[n] != pore) ++changed;
            st->mask[n] = (uint8_t)pore;
            st->phase[n] = 0;
        }
    }
    return changed;
}

/* ------------------------------------------------- cellular-automaton biofilm */
/* The CA block of src/complab.cpp:1453-1715 and its processors:
 *   updateLocalMaskNtotalLattices3D   complab3d_processors_part2.hh:71-212
 *   pushExcessBiomass3D               complab3d_processors_part1.hh:433-660
 *   halfPushExcessBiomass3D           complab3d_processors_part1.hh:662-894
 *   updateAgeDistance3D               complab3d_processors_part2.hh:717-830
 *   createAgeDomain3D                 complab3d_processors_part3.hh:350-370
 * Two orders:
 *   serial = 1: the reference's processors as they run on one block: in-place
 *               traversals (x outer, z inner); a pushing voxel reads its own
 *               biomass as it stands and its neighbours receive their share at
 *               once, capacities come from the total lattice of the sweep's
 *               start; the mask update and the age passes read what earlier
 *               voxels of the same pass wrote.  std::random_shuffle and
 *               std::rand draw, in call order, from ca_seq_next; the
 *               reference's own processors run with the same draws in
 *               oracle/ref/ca_harness.cpp, which pins this order;
 *   serial = 0: the order the CUDA library runs: every voxel plans its
 *               outflows from the sweep's starting state, then every voxel
 *               gathers its own outflows and its neighbours' inflows in
 *               direction order; the draws are the hash of (seed, stream,
 *               site); the mask update reads the previous masks and the age
 *               passes the previous ages (Jacobi). */
#define ORC_CA_THRD 1e-12          /* thrd, src/complab3d_processors.hh:60 (push and loop); the
                                      mask, total and age rules use COMPLAB_THRD */
static const int D6[6][3] = {{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1}};

static uint64_t ca_hash(uint64_t seed, uint64_t stream, uint64_t site) {
    uint64_t z = seed ^ (stream * 0x9E3779B97F4A7C15ull) ^ (site * 0xD1B54A32D192ED03ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
/* the sequential draws of the serial order (one per std::random_shuffle or std::rand call) */
static uint64_t ca_seq_next(const cl_config* cfg, orc_ca* ca) { return ca_hash(cfg->ca_seed, ~0ull, ca->draws++); }
static int ca_wall(const cl_config* c, int m) { return m == c->solid_code || m == c->bb_code; }
static int ca_pore(const cl_config* c, int m) { return in_list(m, c->pore_codes, c->n_pore_codes); }

void orc_ca_init(const cl_config* cfg, const uint8_t* mask, orc_ca* ca) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    int64_t sum = 0;
    for (int x = 0; x < nx; ++x) for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) {
        const int64_t n = site(cfg, x, y, z);
        const int m = mask[n];
        const int wall = ca_wall(cfg, m);
        ca->age[n] = wall ? -1 : (ca_pore(cfg, m) ? 0 : 1);
        ca->distpos[n] = (uint8_t)(!wall && x < nx - 1 && y < ny - 1 && z < nz - 1);
        ca->total[n] = 0.0;
        sum += m;
    }
    ca->sweeps = 0;
    ca->draws = 0;
    ca->mask_sum = sum;
}

/* updateLocalMaskNtotalLattices3D; returns sites whose mask changed, *sum = mask sum */
static int64_t ca_mask_total(const cl_config* cfg, orc_state* st, orc_ca* ca, int64_t* sum, int serial) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, M = cfg->n_microbes;
    const int64_t N = (int64_t)nx * ny * nz;
    const double thrd_mass = cfg->ca_thrd_frac * cfg->ca_bmax;
    uint8_t* nm = serial ? st->mask : (uint8_t*)malloc((size_t)N);
    int64_t changed = 0, s = 0;
    for (int x = 0; x < nx; ++x) for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) {
        const int64_t n = site(cfg, x, y, z);
        const int mk = st->mask[n];
        int out = mk;
        if (!ca_wall(cfg, mk)) {
            double bmass = 0.0;
            int newmask = 0;
            for (int m = 0; m < M; ++m) {
                const double bm = st->bio[(int64_t)m*N + n];
                if (bm > COMPLAB_THRD) { bmass += bm; newmask += cfg->microbe_code[m]; }
            }
            if (fabs(bmass - ca->total[n]) > COMPLAB_THRD) ca->total[n] = bmass;
            const int poreflag = ca_pore(cfg, mk);
            if (!poreflag && bmass < thrd_mass) {
                newmask = cfg->pore_codes[0];
                if (cfg->n_pore_codes > 1) {
                    for (int d = 0; d < 6; ++d) {
                        const int ax = x + D6[d][0], ay = y + D6[d][1], az = z + D6[d][2];
                        if (ax < 0 || ax >= nx || ay < 0 || ay >= ny || az < 0 || az >= nz) continue;
                        const int q = st->mask[site(cfg, ax, ay, az)];
                        if (!ca_wall(cfg, q) && ca_pore(cfg, q)) { newmask = q; break; }
                    }
                }
                out = newmask;
            } else if (poreflag && bmass >= thrd_mass && newmask > 0) {
                out = newmask;
            }
        }
        nm[n] = (uint8_t)out;
        if (out != mk) ++changed;
        s += out;
    }
    if (!serial) { memcpy(st->mask, nm, (size_t)N); free(nm); }
    if (sum) *sum = s;
    return changed;
}

/* the neighbours a voxel may push to, in the reference's order +x -x +y -y +z -z:
 * inside x = 1..nx-2 (bdryGap 1) and the y, z extent (no wrap), not a wall */
static int ca_candidates(const cl_config* cfg, const uint8_t* mask, int x, int y, int z, int* dir, int64_t* q) {
    int nc = 0;
    for (int d = 0; d < 6; ++d) {
        const int ax = x + D6[d][0], ay = y + D6[d][1], az = z + D6[d][2];
        if (ax < 1 || ax > cfg->nx - 2 || ay < 0 || ay >= cfg->ny || az < 0 || az >= cfg->nz) continue;
        const int64_t n = site(cfg, ax, ay, az);
        if (ca_wall(cfg, mask[n])) continue;
        dir[nc] = d; q[nc] = n; ++nc;
    }
    return nc;
}

/* one push sweep */
static void ca_push(const cl_config* cfg, orc_state* st, orc_ca* ca, int serial) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, M = cfg->n_microbes;
    const int64_t N = (int64_t)nx * ny * nz;
    const int half = cfg->ca_half;
    const double Bmax = cfg->ca_bmax;
    const uint64_t sw = ca->sweeps;
    if (!serial) memset(ca->out, 0, sizeof(double) * 6 * M * N);
    for (int x = 1; x <= nx - 2; ++x) for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) {
        const int64_t n = site(cfg, x, y, z);
        const int mk = st->mask[n];
        if (ca_wall(cfg, mk) || (half && ca_pore(cfg, mk))) continue;
        double bMt = ca->total[n];
        if (!(bMt > Bmax)) continue;
        double bMd = half ? bMt * 0.5 : bMt - Bmax;
        if (!half && !(bMd > ORC_CA_THRD)) continue;
        int dir[6]; int64_t q[6];
        const int nc = ca_candidates(cfg, st->mask, x, y, z, dir, q);
        if (nc == 0) continue;            /* boxed in: the excess stays */
        double Bc[CL_MAX_MICROBES];
        for (int m = 0; m < M; ++m) Bc[m] = st->bio[(int64_t)m*N + n];
        int order[6];
        for (int t = 0; t < nc; ++t) order[t] = t;
        if (nc > 1) {
            const uint64_t r = serial ? ca_seq_next(cfg, ca) : ca_hash(cfg->ca_seed, 2 * sw, (uint64_t)n);
            for (int i = nc - 1; i > 0; --i) {
                const int j = (int)((r >> (8 * i)) & 0xff) % (i + 1);
                const int tmp = order[i]; order[i] = order[j]; order[j] = tmp;
            }
        }
        int chk = 0;
        for (int t = 0; t < nc; ++t) {
            const int d = dir[order[t]];
            const int64_t nb = q[order[t]];
            const double nbrbMt = ca_pore(cfg, st->mask[nb]) ? 0.0 : ca->total[nb];
            if (nbrbMt < Bmax) {
                const double cap = Bmax - nbrbMt;
                double partial = bMd;
                if (bMd > cap) { partial = cap; bMd -= cap; }
                else { bMd = 0.0; chk = 1; }
                for (int m = 0; m < M; ++m) {
                    const double cur = serial ? st->bio[(int64_t)m*N + n] : Bc[m];
                    const double shove = cur / bMt * partial;
                    if (shove > ORC_CA_THRD) {
                        if (serial) { st->bio[(int64_t)m*N + n] -= shove; st->bio[(int64_t)m*N + nb] += shove; }
                        else { Bc[m] -= shove; ca->out[((int64_t)d*M + m)*N + n] += shove; }
                    }
                }
                bMt -= partial;
            }
            if (chk) break;
        }
        if (chk) continue;
        /* the rest to one neighbour: the older-age side (age directed), else any */
        int tl[6], nt = 0;
        const int a0 = ca->age[n];
        for (int t = 0; t < nc; ++t) {
            const int a1 = ca->age[q[t]];
            if (half ? a0 >= a1 : a0 > a1) tl[nt++] = t;
        }
        int pk;
        if (serial) {
            /* std::rand() % n with std::rand = the low 31 bits of a draw */
            if (nt > 1) pk = tl[(int)(ca_seq_next(cfg, ca) & 0x7fffffff) % nt];
            else if (nt == 1) pk = tl[0];
            else pk = nc > 1 ? (int)(ca_seq_next(cfg, ca) & 0x7fffffff) % nc : 0;
        } else {
            const uint64_t r = ca_hash(cfg->ca_seed, 2 * sw + 1, (uint64_t)n);
            if (nt > 1) pk = tl[r % (uint64_t)nt];
            else if (nt == 1) pk = tl[0];
            else pk = nc > 1 ? (int)(r % (uint64_t)nc) : 0;
        }
        for (int m = 0; m < M; ++m) {
            const double cur = serial ? st->bio[(int64_t)m*N + n] : Bc[m];
            const double shove = cur / bMt * bMd;
            if (serial) { st->bio[(int64_t)m*N + n] -= shove; st->bio[(int64_t)m*N + q[pk]] += shove; }
            else { Bc[m] -= shove; ca->out[((int64_t)dir[pk]*M + m)*N + n] += shove; }
        }
    }
    if (serial) return;
    for (int x = 0; x < nx; ++x) for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) {
        const int64_t n = site(cfg, x, y, z);
        for (int m = 0; m < M; ++m) {
            double b = st->bio[(int64_t)m*N + n];
            for (int d = 0; d < 6; ++d) b -= ca->out[((int64_t)d*M + m)*N + n];
            for (int d = 0; d < 6; ++d) {
                const int wx = x - D6[d][0], wy = y - D6[d][1], wz = z - D6[d][2];
                if (wx < 1 || wx > nx - 2 || wy < 0 || wy >= ny || wz < 0 || wz >= nz) continue;
                b += ca->out[((int64_t)d*M + m)*N + site(cfg, wx, wy, wz)];
            }
            st->bio[(int64_t)m*N + n] = b;
        }
    }
}

/* one updateAgeDistance3D pass (Jacobi, or in place when serial); returns
 * voxels whose age changed */
static int64_t ca_age_pass(const cl_config* cfg, orc_ca* ca, int serial) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz;
    const int64_t N = (int64_t)nx * ny * nz;
    const double Bmax = cfg->ca_bmax;
    int32_t* na = serial ? ca->age : (int32_t*)malloc(sizeof(int32_t) * (size_t)N);
    int64_t changed = 0;
    for (int x = 0; x < nx; ++x) for (int y = 0; y < ny; ++y) for (int z = 0; z < nz; ++z) {
        const int64_t n = site(cfg, x, y, z);
        const int age = ca->age[n];
        int out = age;
        const double B = ca->total[n];
        if (B > COMPLAB_THRD) {
            int64_t qs[6]; int nq = 0;
            for (int d = 0; d < 6; ++d) {
                const int ax = x + D6[d][0], ay = y + D6[d][1], az = z + D6[d][2];
                if (ax < 0 || ax >= nx || ay < 0 || ay >= ny || az < 0 || az >= nz) continue;
                const int64_t q = site(cfg, ax, ay, az);
                if (ca->distpos[q]) qs[nq++] = q;
            }
            if (age == 0) out = 1;
            else if (age == 1 && (B - Bmax) > -COMPLAB_THRD) {
                int upd = 1;
                for (int t = 0; t < nq; ++t) if (ca->age[qs[t]] == 0) { upd = 0; break; }
                if (upd) out = 2;
            } else {
                int count = 0;
                for (int t = 0; t < nq; ++t)
                    if (ca->age[qs[t]] >= age && (ca->total[qs[t]] - Bmax) > -COMPLAB_THRD) ++count;
                if (count == nq) out = age + 1;
            }
        }
        na[n] = out;
        if (out != age) ++changed;
    }
    if (!serial) { memcpy(ca->age, na, sizeof(int32_t) * (size_t)N); free(na); }
    return changed;
}

static double ca_max_total(const cl_config* cfg, const orc_ca* ca) {
    const int64_t N = (int64_t)cfg->nx * cfg->ny * cfg->nz;
    double mx = ca->total[0];
    for (int64_t n = 1; n < N; ++n) if (ca->total[n] > mx || isnan(ca->total[n])) mx = ca->total[n];
    return mx;
}

int64_t orc_ca_update_mask(const cl_config* cfg, orc_state* st, orc_ca* ca, int serial) {
    int64_t sum = 0;
    const int64_t ch = ca_mask_total(cfg, st, ca, &sum, serial);
    ca->mask_sum = sum;
    return ch;
}

int orc_ca_redistribute(const cl_config* cfg, orc_state* st, orc_ca* ca, int serial,
                        int32_t* sweeps_out, int64_t* changes_out, double* bmax_after) {
    const double Bmax = cfg->ca_bmax;
    int64_t sum = 0;
    int64_t changes = ca_mask_total(cfg, st, ca, &sum, serial);
    double gmax = ca_max_total(cfg, ca);
    if (!isfinite(gmax)) return CL_ERR_DIVERGED;
    int status = CL_OK, sweeps = 0;
    if (gmax - Bmax > ORC_CA_THRD) {
        double prev = gmax;
        int stall = 0;
        for (int64_t wc = 0; gmax - Bmax > ORC_CA_THRD; ++wc) {
            ca_push(cfg, st, ca, serial);
            ca->sweeps += 1;
            ++sweeps;
            changes += ca_mask_total(cfg, st, ca, &sum, serial);
            gmax = ca_max_total(cfg, ca);
            if (gmax > prev - ORC_CA_THRD) { if (++stall >= 100) { status = CL_WARN_NOT_CONVERGED; break; } }
            else stall = 0;
            prev = gmax;
            if (wc % 50 == 0) {
                int64_t ch = 1;
                int passes = 0;
                while (ch != 0) {
                    ch = ca_age_pass(cfg, ca, serial);
                    if (++passes > 1000) break;
                }
                if (ch != 0) { status = CL_WARN_NOT_CONVERGED; break; }
            }
            if (wc > 1000) { status = CL_WARN_NOT_CONVERGED; break; }
        }
    }
    if (sum != ca->mask_sum) {
        ca_age_pass(cfg, ca, serial);
        ca->mask_sum = sum;
    }
    if (sweeps_out) *sweeps_out = sweeps;
    if (changes_out) *changes_out = changes;
    if (bmax_after) *bmax_after = gmax;
    return status;
}

/* ---------------------------------------------------------------- MLP (FP64) */
static double gelu(double v) { return 0.5 * v * (1.0 + erf(v / sqrt(2.0))); }
static double gelu_d(double v) {
    return 0.5 * (1.0 + erf(v / sqrt(2.0))) + v * exp(-0.5 * v * v) / sqrt(2.0 * M_PI);
}

/* Forward and analytic backward of a 2-hidden-layer GELU MLP with MSE loss,
 * following the structure of surrogate_training/trainSurrogate.py:132-166
 * (tanh hidden layers there, GELU here). */
double orc_mlp_forward_backward(int n_in, int H, int n_out, const double* p,
                                const double* xin, const double* yin, int n,
                                double* grads, double* y_hat) {
    const double* W1 = p;               const double* b1 = W1 + H*n_in;
    const double* W2 = b1 + H;          const double* b2 = W2 + H*H;
    const double* W3 = b2 + H;          const double* b3 = W3 + n_out*H;
    int np = H*n_in + H + H*H + H + n_out*H + n_out;
    if (grads) memset(grads, 0, sizeof(double) * np);
    double* gW1 = grads; double* gb1 = grads ? gW1 + H*n_in : NULL;
    double* gW2 = grads ? gb1 + H : NULL; double* gb2 = grads ? gW2 + H*H : NULL;
    double* gW3 = grads ? gb2 + H : NULL; double* gb3 = grads ? gW3 + n_out*H : NULL;
    double loss = 0.0;
    double z1[256], a1[256], z2[256], a2[256], yo[64], dy[64], d2[256], d1[256];
    for (int k = 0; k < n; ++k) {
        const double* x = xin + (int64_t)k*n_in;
        for (int h = 0; h < H; ++h) {
            double s = b1[h]; for (int i = 0; i < n_in; ++i) s += W1[h*n_in + i]*x[i];
            z1[h] = s; a1[h] = gelu(s);
        }
        for (int h = 0; h < H; ++h) {
            double s = b2[h]; for (int i = 0; i < H; ++i) s += W2[h*H + i]*a1[i];
            z2[h] = s; a2[h] = gelu(s);
        }
        for (int o = 0; o < n_out; ++o) {
            double s = b3[o]; for (int i = 0; i < H; ++i) s += W3[o*H + i]*a2[i];
            yo[o] = s;
            if (y_hat) y_hat[(int64_t)k*n_out + o] = s;
            double e = s - yin[(int64_t)k*n_out + o];
            loss += e*e;
            dy[o] = 2.0 * e / ((double)n * n_out);
        }
        if (!grads) continue;
        for (int o = 0; o < n_out; ++o) {
            gb3[o] += dy[o];
            for (int i = 0; i < H; ++i) gW3[o*H + i] += dy[o]*a2[i];
        }
        for (int h = 0; h < H; ++h) {
            double s = 0; for (int o = 0; o < n_out; ++o) s += W3[o*H + h]*dy[o];
            d2[h] = s * gelu_d(z2[h]);
        }
        for (int h = 0; h < H; ++h) {
            gb2[h] += d2[h];
            for (int i = 0; i < H; ++i) gW2[h*H + i] += d2[h]*a1[i];
        }
        for (int h = 0; h < H; ++h) {
            double s = 0; for (int o = 0; o < H; ++o) s += W2[o*H + h]*d2[o];
            d1[h] = s * gelu_d(z1[h]);
        }
        for (int h = 0; h < H; ++h) {
            gb1[h] += d1[h];
            for (int i = 0; i < n_in; ++i) gW1[h*n_in + i] += d1[h]*x[i];
        }
    }
    return loss / ((double)n * n_out);
}

/* --------------------------------------------------------- surrogate (FP64) */
/* defineSurrogateModel (surrogateModel.hh:390-430): mapminmax input
 * xs = (x - offset)*gain + ymin, tansig hidden layers, linear output, reverse
 * map y = (a - ymin)/gain + offset.  Inputs are first clamped to [x_lo, x_hi]. */
void orc_surrogate_forward(const cl_surrogate_net* net, const double* xin, double* yout, int64_t n) {
    int L = net->n_layers;
    for (int64_t k = 0; k < n; ++k) {
        double a[CL_SRG_MAX_WIDTH], b[CL_SRG_MAX_WIDTH];
        int w0 = net->widths[0];
        for (int i = 0; i < w0; ++i) {
            double v = xin[k*w0 + i];
            if (v < net->x_lo[i]) v = net->x_lo[i];
            if (v > net->x_hi[i]) v = net->x_hi[i];
            a[i] = (v - net->x_offset[i]) * net->x_gain[i] + net->x_ymin;
        }
        const double* p = net->params;
        for (int l = 0; l < L; ++l) {
            int wi = net->widths[l], wo = net->widths[l + 1];
            const double* W = p; const double* bb = p + wo*wi;
            for (int o = 0; o < wo; ++o) {
                double s = 0.0;
                for (int i = 0; i < wi; ++i) s += W[o*wi + i] * a[i];
                s += bb[o];
                b[o] = (l < L - 1) ? (2.0 / (1.0 + exp(-2.0 * s)) - 1.0) : s;
            }
            for (int o = 0; o < wo; ++o) a[o] = b[o];
            p += wo*wi + wo;
        }
        int wl = net->widths[L];
        for (int o = 0; o < wl; ++o)
            yout[k*wl + o] = (a[o] - net->y_ymin) / net->y_gain[o] + net->y_offset[o];
    }
}

/* fdDiffusion3D (src/complab3d_processors_part2.hh:258-420): one explicit
 * finite-difference step of the sessile biomass of the microbes in sel on the
 * sites of x = 1 .. nx-2 whose material number exceeds 1, reading a copy
 * taken before the step; the boundary tests in the reference's order (the
 * upstream side first); values below COMPLAB_THRD read as zero; a result not
 * above COMPLAB_THRD leaves the biomass as it was; a neighbour outside the
 * lattice reads zero. */
void orc_fd_diffuse(const cl_config* cfg, orc_state* st, double nu, uint32_t sel) {
    const int nx = cfg->nx, ny = cfg->ny, nz = cfg->nz, M = cfg->n_microbes;
    const int64_t N = (int64_t)nx * ny * nz;
    double* cp = (double*)malloc(sizeof(double) * (size_t)(M > 0 ? M : 1) * (size_t)N);
    memcpy(cp, st->bio, sizeof(double) * (size_t)M * (size_t)N);
    const uint8_t* mk = st->mask;
    for (int x = 1; x <= nx - 2; ++x)
        for (int y = 0; y < ny; ++y)
            for (int z = 0; z < nz; ++z) {
                const int64_t n = site(cfg, x, y, z);
                if (mk[n] <= 1) continue;
                int mxp = 0, mxn = 0, myp = 0, myn = 0, mzp = 0, mzn = 0;
                if (x == 1) mxp = mk[site(cfg, x + 1, y, z)];
                else if (x == nx - 2) mxn = mk[site(cfg, x - 1, y, z)];
                else { mxp = mk[site(cfg, x + 1, y, z)]; mxn = mk[site(cfg, x - 1, y, z)]; }
                if (y == 0) { if (y + 1 < ny) myp = mk[site(cfg, x, y + 1, z)]; }
                else if (y == ny - 1) myn = mk[site(cfg, x, y - 1, z)];
                else { myp = mk[site(cfg, x, y + 1, z)]; myn = mk[site(cfg, x, y - 1, z)]; }
                if (z == 0) { if (z + 1 < nz) mzp = mk[site(cfg, x, y, z + 1)]; }
                else if (z == nz - 1) mzn = mk[site(cfg, x, y, z - 1)];
                else { mzp = mk[site(cfg, x, y, z + 1)]; mzn = mk[site(cfg, x, y, z - 1)]; }
                for (int m = 0; m < M; ++m) {
                    if (!((sel >> m) & 1u)) continue;
                    const double* c = cp + (int64_t)m * N;
#define FD_AT(xx, yy, zz) (((xx) >= 0 && (xx) < nx && (yy) >= 0 && (yy) < ny && (zz) >= 0 && (zz) < nz) ? c[site(cfg, xx, yy, zz)] : 0.0)
                    double b0 = c[n], bxp, bxn, byp, byn, bzp, bzn;
                    if (x == 1 || mxn < 2) { bxp = FD_AT(x + 1, y, z); bxn = b0; }
                    else if (x == nx - 2 || mxp < 2) { bxp = b0; bxn = FD_AT(x - 1, y, z); }
                    else { bxp = FD_AT(x + 1, y, z); bxn = FD_AT(x - 1, y, z); }
                    if (y == 0 || myn < 2) { byp = FD_AT(x, y + 1, z); byn = b0; }
                    else if (y == ny - 1 || myp < 2) { byp = b0; byn = FD_AT(x, y - 1, z); }
                    else { byp = FD_AT(x, y + 1, z); byn = FD_AT(x, y - 1, z); }
                    if (z == 0 || mzn < 2) { bzp = FD_AT(x, y, z + 1); bzn = b0; }
                    else if (z == nz - 1 || mzp < 2) { bzp = b0; bzn = FD_AT(x, y, z - 1); }
                    else { bzp = FD_AT(x, y, z + 1); bzn = FD_AT(x, y, z - 1); }
#undef FD_AT
                    if (b0 < COMPLAB_THRD) b0 = 0;
                    if (bxp < COMPLAB_THRD) bxp = 0;
                    if (bxn < COMPLAB_THRD) bxn = 0;
                    if (byp < COMPLAB_THRD) byp = 0;
                    if (byn < COMPLAB_THRD) byn = 0;
                    if (bzp < COMPLAB_THRD) bzp = 0;
                    if (bzn < COMPLAB_THRD) bzn = 0;
                    const double nb = b0 + nu * ((bxp - 2 * b0 + bxn) + (byp - 2 * b0 + byn) + (bzp - 2 * b0 + bzn));
                    if (nb > COMPLAB_THRD) st->bio[(int64_t)m * N + n] = nb;
                }
            }
    free(cp);
}
