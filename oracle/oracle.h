/*
 * oracle.h -- FP64 CPU oracle for the CompLB3D hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * legs of bench.py load this library, and only as the checker or the timed CPU
 * baseline.  The product path (the CUDA library) never calls it.
 *
 * It restates, processor by processor and in the reference's order, the
 * per-timestep loop of src/complab.cpp:1152-1860 over full-lattice FP64 arrays
 * with two-buffer push streaming.  Palabos v2.3.0 (the third-party library that
 * holds the lattice arithmetic: IncBGKdynamics, AdvectionDiffusionBGKdynamics,
 * BounceBack, NoDynamics, the regularized local pressure boundary, the
 * advection-diffusion Dirichlet boundary, FlatAdiabaticBoundaryFunctional3D and
 * util::ValueTracer) is not vendored with the reference, so those parts are a
 * restatement of Palabos's published algorithms: PARITY UNPINNED against
 * Palabos itself.  The reference's own Palabos-free code (PCF+AA speciation,
 * the surrogate network header, the example rate-law headers) is compiled from
 * its sources into oracle/_ref and pins the restated parts that have a
 * counterpart there.
 *
 * Storage: flow populations as deviations fbar_i = f_i - t_i, layout [19][N];
 * solute populations g_i (full), layout [7][N] per solute; site
 * n = (x*ny + y)*nz + z; y and z periodic.
 */
#ifndef COMPLAB_ORACLE_H
#define COMPLAB_ORACLE_H
#include <stdint.h>
#include "../include/complab_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* node classes */
#define ORC_NODYN 0
#define ORC_BB    1
#define ORC_FLUID 2   /* NS: IncBGK(omega); ADE: omega_pore */
#define ORC_BIO   3   /* NS: IncBGK(omega_bio); ADE: omega_bio */

int  orc_config_size(void);
void orc_classes_from_mask(const cl_config* cfg, const uint8_t* mask,
                           uint8_t* ns_class, uint8_t* ade_class);

/* ---- flow ---------------------------------------------------------------- */
void   orc_flow_init(const cl_config* cfg, const uint8_t* ns_class, double* f);
/* one collideAndStream; returns the average energy 0.5*<|j|^2> over BGK cells */
double orc_flow_step(const cl_config* cfg, const uint8_t* ns_class,
                     const double* f_in, double* f_out);
/* collideAndStream until ValueTracer(1,1000,eps) converges or max_it;
 * returns the reference's iT at exit, -1 on divergence (NaN). */
int    orc_flow_solve(const cl_config* cfg, const uint8_t* ns_class, double* f,
                      double* f_tmp, int max_it, double eps, double* energy_hist);
/* density and velocity of every site, as Palabos computeDensity/computeVelocity */
void   orc_flow_macro(const cl_config* cfg, const uint8_t* ns_class, const double* f,
                      double* rho, double* u /*[3][N]*/);

/* ---- transport ------------------------------------------------------------ */
typedef struct {
    double*  g;        /* [S][7][N] mobile solute populations (immobile slots unused) */
    double*  g_tmp;    /* same size, streaming target */
    double*  imm;      /* [S][N] immobile solute inventories (mobile slots unused) */
    double*  bio;      /* [M][N] sessile biomass */
    double*  u;        /* [3][N] coupled velocity */
    uint8_t* mask;     /* [N] */
    uint8_t* ade_class;/* [N] */
    double*  rho_bc;   /* [S][2][ny*nz] prescribed boundary density (0: x=0, 1: x=nx-1) */
    int32_t* eq_iters; /* [N] Newton iterations of the last equilibrium step (may be NULL) */
    const cl_surrogate_net* srg_nets;  /* [CL_MAX_SRG_ORG] networks of the surrogate organisms (may be NULL) */
    uint8_t* phase;    /* [N] dissolvable phase id, 0 = none (may be NULL without dissolution) */
    /* compiled rate laws standing in for the rate table (NULL: the table):
     * kin(B, nB, C, nC, subsR, bioR, mask) and abio(C, nC, subsR, mask), the
     * defineRxnKinetics / defineAbioticRxnKinetics signatures over arrays */
    void (*kin)(const double*, int, const double*, int, double*, double*, int);
    void (*abio)(const double*, int, double*, int);
} orc_state;

void orc_ade_init(const cl_config* cfg, orc_state* st);
/* one transport step; returns the number of Newton solves that did not converge */
int64_t orc_transport_step(const cl_config* cfg, orc_state* st);
/* its reaction stage alone (kinetics .. equilibrium on the current densities) */
int64_t orc_reaction_stage(const cl_config* cfg, orc_state* st);
/* the step in its three parts: orc_transport_step = orc_collide, then
 * orc_reaction_stage, then orc_stream; orc_reaction_ops runs the processors
 * selected by ops (kinetics and surrogate share one increment lattice, as
 * run_kinetics and run_surrogate3D share dC; abiotic includes dissolution) */
#define ORC_OP_KINETICS    1
#define ORC_OP_SURROGATE   2
#define ORC_OP_ABIOTIC     4
#define ORC_OP_EQUILIBRIUM 8
#define ORC_OP_ALL         15
void    orc_collide(const cl_config* cfg, orc_state* st);
int64_t orc_reaction_ops(const cl_config* cfg, orc_state* st, int ops);
void    orc_stream(const cl_config* cfg, orc_state* st);
/* solute density of every site (mobile: sum of g; immobile: inventory) */
void orc_solute_density(const cl_config* cfg, const orc_state* st, int s, double* out);

/* table-driven rate law, one voxel (mirrors defineRxnKinetics / defineAbioticRxnKinetics) */
void orc_rates(const cl_config* cfg, int abiotic, const double* C, const double* B,
               double* subsR, double* bioR);

/* geometry updates (precipNodeConversion3D, dissolNodeConversion3D);
 * return the number of sites whose mask changed */
int64_t orc_precip_convert(const cl_config* cfg, orc_state* st);
int64_t orc_dissol_convert(const cl_config* cfg, orc_state* st);

/* ---- cellular-automaton biofilm -------------------------------------------- */
typedef struct {
    double*  total;    /* [N] total biomass */
    int32_t* age;      /* [N] age wavefront */
    uint8_t* distpos;  /* [N] distance field positive */
    double*  out;      /* [6][M][N] outflows of one sweep (order serial = 0) */
    uint64_t sweeps;
    int64_t  mask_sum;
    uint64_t draws;    /* sequential draws taken (serial order) */
} orc_ca;
void    orc_ca_init(const cl_config* cfg, const uint8_t* mask, orc_ca* ca);
/* serial = 1: the reference's in-place processor order; 0: plan then gather */
int64_t orc_ca_update_mask(const cl_config* cfg, orc_state* st, orc_ca* ca, int serial);
int     orc_ca_redistribute(const cl_config* cfg, orc_state* st, orc_ca* ca, int serial,
                            int32_t* sweeps, int64_t* mask_changes, double* bmax_after);
/* fdDiffusion3D: one finite-difference step of the sessile biomass of the microbes in sel */
void    orc_fd_diffuse(const cl_config* cfg, orc_state* st, double nu, uint32_t sel);

/* ---- speciation ------------------------------------------------------------ */
/* totals from species (calc_component_totals) */
void orc_eq_totals(const cl_eq_system* sys, const double* species, double* totals);
/* cold start of the reference (solve_equilibrium_anderson:977-994) */
void orc_eq_cold_start(const cl_eq_system* sys, const double* species, double* x0);
/* FP64 Newton in log10 free components.  Returns iterations used; *converged. */
int  orc_eq_newton(const cl_eq_system* sys, const double* totals, double* x,
                   int max_iter, double tol, int* converged);
double orc_eq_residual(const cl_eq_system* sys, const double* totals, const double* x);
void orc_eq_species(const cl_eq_system* sys, const double* x, double* c);
/* batch: start = CL_EQ_START_COLD uses cold_species, else x_io is the start */
void orc_eq_batch(const cl_eq_system* sys, const double* totals, const double* cold_species,
                  double* x_io, int32_t* iters, uint8_t* status, int64_t n, int start);
/* the reference's live solver (PCF + Anderson), calculate_species_concentrations */
int  orc_pcf_solve(const cl_eq_system* sys, const double* species_in, double* species_out, int* iters);
void orc_pcf_batch(const cl_eq_system* sys, const double* species_in, double* species_out, int32_t* iters,
                   uint8_t* conv, int64_t n);

/* ---- MLP n_in -> H -> H -> n_out, GELU, FP64 (gradient oracle) ------------ */
/* params packed: W1[H][n_in] b1[H] W2[H][H] b2[H] W3[n_out][H] b3[n_out];
 * loss = mean over samples and outputs of (y_hat - y)^2 */
double orc_mlp_forward_backward(int n_in, int H, int n_out, const double* params,
                                const double* x, const double* y, int n,
                                double* grads /* may be NULL */, double* y_hat /* may be NULL */);

/* ---- surrogate network forward (defineSurrogateModel), FP64 ----------------- */
void orc_surrogate_forward(const cl_surrogate_net* net, const double* x, double* y, int64_t n);

#ifdef __cplusplus
}
#endif
#endif
