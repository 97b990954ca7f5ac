/*
 * complab_gpu.h -- C ABI of the B200 (sm_100a) implementation of CompLB3D's
 * per-timestep hot path.
 *
 * The reference drives its hot path through Palabos data processors
 * (`applyProcessingFunctional(new X(...), box, latticeVector)`,
 * src/complab.cpp:1152-1860) over FP64 AoS lattices.  This header replaces
 * that processor surface with plain C entry points over a device-resident
 * context: plain pointers and sizes, no C++ or torch types, an int status on
 * every call (0 = ok, < 0 = error, > 0 = soft warning such as "some Newton
 * solves fell back or did not converge").  Nothing traps on the device; every
 * device loop is bounded and reports through a status word.
 *
 * Data conventions
 *   - Site index n = (x*ny + y)*nz + z   (x slowest, z fastest).  This is the
 *     reader order of the reference's geometry file (x-slices, each slice
 *     y-major then z; src/complab_functions.hh:127-156).
 *   - nx INCLUDES the inlet (x=0) and outlet (x=nx-1) planes, as the reference
 *     does after `nx += 2` (src/complab_functions.hh:769).
 *   - y and z are periodic.
 *   - Host buffers are owned by the caller, device memory by the context.
 *   - All calls are synchronous on the context's stream unless they say
 *     otherwise.  One context per GPU; a context is not thread-safe.
 */
#ifndef COMPLAB_GPU_H
#define COMPLAB_GPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CL_MAX_SOLUTES   32
#define CL_MAX_MICROBES  12
#define CL_MAX_RXN       16
#define CL_MAX_MONOD     3
#define CL_MAX_COMP      24      /* tableau components (batch speciation); the transport step takes 1..5 */
#define CL_MAX_SPECIES   128     /* tableau species (batch speciation); the transport step: one per solute */
#define CL_MAX_CODES     8
#define CL_MAX_PHASES    4

/* status codes */
#define CL_OK                 0
#define CL_WARN_NOT_CONVERGED 1   /* soft: a bounded loop ended before its tolerance */
#define CL_ERR_ARG          (-1)  /* bad argument (null pointer, size out of range) */
#define CL_ERR_CUDA         (-2)  /* a CUDA runtime call failed */
#define CL_ERR_STATE        (-3)  /* call out of order (e.g. step before mask upload) */
#define CL_ERR_NOMEM        (-4)  /* device allocation failed */
#define CL_ERR_DIVERGED     (-5)  /* NaN in a convergence tracer (reference: "simulation diverged") */

/* boundary types of a solute on an x face (reference <left_boundary_type>) */
#define CL_BC_DIRICHLET   0
#define CL_BC_NEUMANN     1       /* zero gradient: FlatAdiabaticBoundaryFunctional3D */

/* One table-driven rate expression.  It covers the shipped example rate laws
 * (e.g. examples/05_biotic_cellular_automaton/defineKinetics.hh:57-86,
 *  examples/13_precipitation/defineAbioticKinetics.hh:39-58) and the dual-Monod
 * law of the 128^3 biotic workload:
 *   r = k * (B_m if microbe >= 0) * prod_j C[monod_s[j]]/(Ks[j] + C[monod_s[j]])
 *         * P,   P = prod_j C[mass_s[j]]
 *   subsR[s] += nu[s] * r ;  bioR[microbe] += yield * r
 * With ksp > 0 the mass-action factor P becomes the saturation-index drive
 * max(P / ksp - 1, 0) (precipitation at a rate k (Omega - 1) above
 * saturation; an extension: the reference has no solubility products). */
typedef struct {
    int32_t microbe;                   /* -1 = abiotic */
    int32_t n_monod;
    int32_t monod_s[CL_MAX_MONOD];
    double  monod_ks[CL_MAX_MONOD];
    int32_t n_mass;
    int32_t mass_s[2];
    double  k;
    double  nu[CL_MAX_SOLUTES];
    double  yield;
    double  ksp;                       /* > 0: saturation-index drive on the mass-action product */
} cl_rxn;

/* Components-and-species tableau (reference EquilibriumChemistry<T>,
 * src/complab3d_processors_part4_eqsolver.hh:186-1271).  In the transport
 * step the species are the solutes in order (1..5 components); the batch
 * solver takes up to CL_MAX_COMP components over CL_MAX_SPECIES species (the
 * reference's uranium network is 17 x 95).  Rows of all zeros are
 * non-equilibrium species.
 * solver selects the equilibrium solve of the transport step:
 *   CL_EQ_SOLVER_NEWTON  Newton in log10 free components (the reference's
 *                        reserve solver, NR_reserve.hh:512-615, with the
 *                        safeguards listed in the design notes); a voxel whose
 *                        solve does not converge is left unchanged;
 *   CL_EQ_SOLVER_PCF     the reference's live solver: positive continued
 *                        fractions with Anderson acceleration
 *                        (solve_equilibrium_anderson, part4_eqsolver.hh:952-1172;
 *                        convergence ||f||_2 < tol on the PCF correction, at most
 *                        max_iter iterations, depth anderson_depth (0: 4, the
 *                        setting of complab.cpp:425), condition limit 1e10,
 *                        mixing 1); its result is applied whether or not it
 *                        converged, as run_equilibrium_biotic applies it. */
#define CL_EQ_SOLVER_NEWTON 0
#define CL_EQ_SOLVER_PCF    1
typedef struct {
    int32_t n_comp;
    int32_t n_species;                 /* == number of solutes it acts on */
    int32_t comp_species[CL_MAX_COMP]; /* species index named like component j, or -1 */
    double  stoich[CL_MAX_SPECIES][CL_MAX_COMP];
    double  logk[CL_MAX_SPECIES];
    int32_t max_iter;                  /* Newton iterations (cold); PCF iterations */
    double  tol;                       /* Newton: relative mass-balance residual; PCF: ||f||_2 */
    int32_t warm_iter;                 /* k: Newton iterations allowed from the learned start */
    int32_t solver;                    /* CL_EQ_SOLVER_* of the transport step */
    int32_t anderson_depth;            /* PCF history depth (0: 4) */
} cl_eq_system;

/* Dissolvable solid phase (reference SolidPhase, src/dissolutionVOP.hh:142-154)
 * and its rate law (the defineDissolutionRate hook, defineAbioticKinetics.hh:292):
 *   rate = k * mineral * prod_j water[mass_s[j]]   (water: mean over open faces)
 *   mineralR = -rate ;  subsR[s] = nu[s] * rate
 * as examples/14_dissolution and 15_precip_and_dissolution write it (calcite or
 * FeS + H+).  phases[k].id must be k+1 (the reference numbers them so,
 * complab.cpp:329); the substrate must be an immobile solute. */
typedef struct {
    int32_t id;                        /* 1-based */
    int32_t material;                  /* material number the phase occupies (grain phases) */
    int32_t substrate;                 /* immobile solute holding its inventory */
    int32_t is_precipitate;            /* stamped by precipitation instead of seeded from the geometry */
    double  full_density;              /* mol/L in a full voxel */
    double  initial_fill;              /* mol/L seeded on `material` at start */
    double  k;
    int32_t n_mass;
    int32_t mass_s[2];
    double  nu[CL_MAX_SOLUTES];
} cl_phase;

/* ---- surrogate reaction type ----------------------------------------
 * Feed-forward network with mapminmax scaling (reference defineSurrogateModel,
 * surrogateModel.hh:252-501).  Layers: widths[0] inputs ... widths[n_layers]
 * outputs; tanh on hidden layers, linear output. */
#define CL_SRG_MAX_LAYERS 5
#define CL_SRG_MAX_WIDTH  32
typedef struct {
    int32_t n_layers;
    int32_t widths[CL_SRG_MAX_LAYERS + 1];
    double  x_offset[CL_SRG_MAX_WIDTH], x_gain[CL_SRG_MAX_WIDTH], x_ymin;
    double  y_offset[CL_SRG_MAX_WIDTH], y_gain[CL_SRG_MAX_WIDTH], y_ymin;
    double  x_lo[CL_SRG_MAX_WIDTH], x_hi[CL_SRG_MAX_WIDTH];   /* input clamp box */
    /* weights, row-major W[l][out][in] then bias b[l][out], packed layer by layer */
    double  params[4096];
} cl_surrogate_net;
/* One organism of the surrogate reaction type (run_surrogate3D,
 * src/complab3d_processors_surrogate.hh:74-295).  Per voxel where its biomass
 * exceeds 1e-12: Michaelis-Menten uptake estimates Fin[s] = Vmax*C/(Kc+C) (or,
 * with no Vmax, the flux that would exhaust C in one step), capped by that
 * exhaustion flux; the network maps its inputs to a growth rate (1/h) and,
 * optionally, uptake fluxes Fout[s] (default Fout = Fin); biomass grows by
 * mu*B*dt/3600 or decays by kd*B*dt; the substrate draw summed over organisms is
 * clamped to what the voxel holds.  Fluxes are mmol/gDW/h, B mol/L. */
#define CL_MAX_SRG_ORG     2
#define CL_SRG_IN_FIN      0     /* input: Fin of solute in_index */
#define CL_SRG_IN_CONC     1     /* input: concentration of solute in_index */
#define CL_SRG_IN_BIOMASS  2     /* input: this organism's biomass */
#define CL_SRG_OUT_GROWTH  0     /* output: specific growth rate, 1/h */
#define CL_SRG_OUT_FOUT    1     /* output: uptake flux of solute out_index (positive = consumed) */
typedef struct {
    int32_t microbe;                       /* biomass field of this organism */
    int32_t net;                           /* network slot set by cl_set_surrogate */
    int32_t in_kind[CL_SRG_MAX_WIDTH], in_index[CL_SRG_MAX_WIDTH];
    int32_t out_kind[CL_SRG_MAX_WIDTH], out_index[CL_SRG_MAX_WIDTH];
    double  kc[CL_MAX_SOLUTES];            /* half-saturation per solute */
    double  vmax[CL_MAX_SOLUTES];          /* <maximum_uptake_flux>; <= 1e-12: exhaustion flux */
    double  mw;                            /* <biomass_molar_mass>, gDW/mol */
    double  kd;                            /* decay, 1/s */
} cl_srg_organism;

typedef struct {
    /* lattice */
    int32_t nx, ny, nz;
    /* material numbers (reference <material_numbers>) */
    int32_t solid_code;                /* NoDynamics (<solid>) */
    int32_t bb_code;                   /* BounceBack (<bounce_back>) */
    int32_t n_pore_codes;
    int32_t pore_codes[CL_MAX_CODES];
    int32_t n_bio_codes;
    int32_t bio_codes[CL_MAX_CODES];
    /* flow (D3Q19 incompressible BGK) */
    double  tau_ns;
    double  perm_ratio;                /* biofilm permeability ratio X (<= 1e-14: biofilm is bounce-back) */
    double  rho_in, rho_out;           /* densities at x=0 and x=nx-1 */
    /* solutes (D3Q7 advection-diffusion BGK) */
    int32_t n_solutes;
    double  omega_pore[CL_MAX_SOLUTES];
    double  omega_bio[CL_MAX_SOLUTES];
    int32_t immobile[CL_MAX_SOLUTES];
    int32_t left_type[CL_MAX_SOLUTES], right_type[CL_MAX_SOLUTES];
    double  left_value[CL_MAX_SOLUTES], right_value[CL_MAX_SOLUTES];
    double  c0[CL_MAX_SOLUTES];
    /* sessile biomass, one scalar field per microbe */
    int32_t n_microbes;
    double  b_max;                     /* <max_biomass_density> (CA trigger) */
    double  thrd_bfilm_frac;           /* <thrd_biofilm_fraction> */
    double  dt;                        /* ade_dt, seconds per transport step */
    /* reactions */
    int32_t enable_kinetics;
    int32_t enable_abiotic;
    int32_t abiotic_surface_only;      /* <precipitation><surface_only> */
    int32_t n_rxn;
    cl_rxn  rxn[CL_MAX_RXN];
    double  decay[CL_MAX_MICROBES];    /* kd, 1/s */
    int32_t use_equilibrium;
    cl_eq_system eq;
    int32_t eq_warm_previous;          /* 1: start each voxel's Newton from its previous converged solutions
                                          (the linear extrapolation of the last two; cold start after
                                          eq.warm_iter misses); 0: the reference's cold start */
    /* precipitation / dissolution (reference src/precipitationVOP.hh, src/dissolutionVOP.hh) */
    int32_t precip_enabled;
    int32_t precip_substrate;          /* immobile solute holding the precipitate */
    double  max_precip_rho;
    int32_t precip_code;               /* mask code a full voxel becomes */
    int32_t precip_phase_id;
    int32_t dissol_enabled;
    double  reopen_fraction;
    int32_t dissol_surface_only;
    int32_t dissol_apply_at_walls;     /* 0: as the reference, a mineral decrement on a solid/bounce-back
                                          voxel is dropped (update_abiotic_rxnLattices skips walls);
                                          1: it is applied, so grains can dissolve and reopen */
    int32_t n_phases;
    cl_phase phases[CL_MAX_PHASES];
    /* surrogate reaction type: organisms, networks uploaded by cl_set_surrogate */
    int32_t n_srg;
    cl_srg_organism srg[CL_MAX_SRG_ORG];
    /* cellular-automaton biofilm: <microbiology> maximum_biomass_density,
     * thrd_biofilm_fraction, CA_method; the biofilm material of each microbe
     * (bio_dynamics[m][0]); the seed of the counter-based generator that stands
     * for std::rand / std::random_shuffle */
    int32_t ca_enabled;
    int32_t ca_half;                   /* CA_method "half": halfPushExcessBiomass3D */
    double  ca_bmax;
    double  ca_thrd_frac;
    int32_t microbe_code[CL_MAX_MICROBES];
    uint64_t ca_seed;
    /* the rate laws: CL_RATELAW_TABLE runs the rxn table above; a compiled law
     * (include/complab_ratelaw.hpp) replaces the table as the reference's
     * compiled defineKinetics.hh / defineAbioticKinetics.hh do:
     *   CL_RATELAW_ZHAO  the reference's default Zhao uranium / iron / sulfur
     *                    network, on its 24-substrate layout (speciation off)
     *                    with 12 sessile biomass pools; substrates 2, 4, 5, 6,
     *                    9, 13, 21, 22, 23 immobile */
    int32_t rate_law;
    /* microbes solved by LBM (the reference's planktonic biomass, solver_type
     * LBM: soluteDomainSetup of a bFree lattice, complab.cpp:788-797): 0 =
     * sessile (the FP64 biomass field); s + 1 = the microbe's biomass is the
     * density of mobile solute s, which carries its transport and boundary
     * conditions; the kinetics read it and add the microbe's growth to it.
     * Table rate laws only; no surrogate organisms or CA on such a microbe. */
    int32_t microbe_carrier[CL_MAX_MICROBES];
} cl_config;
#define CL_RATELAW_TABLE 0
#define CL_RATELAW_ZHAO  1

typedef struct cl_ctx cl_ctx;

/* ---- context ---------------------------------------------------------------
 * Replaces the lattice construction of src/complab.cpp:588-884 and the dynamics
 * assignment of NSdomainSetup / soluteDomainSetup (src/complab_functions.hh:245-340).
 * `stream` is a cudaStream_t (may be NULL: the context creates its own). */
cl_ctx* cl_create(const cl_config* cfg, void* stream, int* status);
int     cl_destroy(cl_ctx* ctx);
const char* cl_last_error(void);
int     cl_device_bytes(const cl_ctx* ctx, uint64_t* bytes);
/* sizeof of the ABI structs, for binding checks: [cl_config, cl_rxn,
 * cl_eq_system, cl_phase, cl_surrogate_net]; returns how many were written */
int     cl_abi_sizes(int32_t* sizes, int32_t n);
/* the FP64 10^x the Newton solves use (which = 0) or CUDA's exp10 (which = 1)
 * on n host values, for accuracy checks; no counterpart in the reference */
int     cl_math_exp10(const double* x, double* y, int64_t n, int32_t which);

/* geometry: one material number per site, 0..255 (readGeometry, src/complab_functions.hh:127-156) */
int cl_upload_mask(cl_ctx* ctx, const uint8_t* mask);
int cl_download_mask(cl_ctx* ctx, uint8_t* mask);

/* ---- flow -------------------------------------------------------------------
 * cl_flow_init:  initializeAtEquilibrium with the linear PressureGradient profile
 *                (src/complab_functions.hh:72-84,285-290).
 * cl_flow_steps: n collideAndStream steps (src/complab.cpp:607-620).
 * cl_flow_solve: collideAndStream until the ValueTracer(1, 1000, eps) on the
 *                average energy converges, at most max_it steps
 *                (src/complab.cpp:593,607-611).  *iters = the step index at
 *                which it converged (reference's iT), or max_it.
 * cl_couple_velocity: latticeToPassiveAdvDiff (src/complab.cpp:1097-1109). */
int cl_flow_init(cl_ctx* ctx);
int cl_flow_steps(cl_ctx* ctx, int32_t n);
int cl_flow_solve(cl_ctx* ctx, int32_t max_it, double eps, int32_t* iters);
int cl_flow_energy(cl_ctx* ctx, double* energy);
int cl_couple_velocity(cl_ctx* ctx);
/* NS dynamics switch after a mask change (updateNsLatticesDynamics3D,
 * src/complab3d_processors_part2.hh:630-695) and the solute omega switch
 * (updateSoluteDynamics3D, :461-529). */
int cl_update_dynamics(cl_ctx* ctx);

/* The host driver's Peclet calibration (src/complab.cpp:641-669):
 * cl_flow_velocity_stats returns computeAverage(velocityNorm) and
 * computeMax(u_x) over x = 1..nx-2 and computeAverage(u_x) over the plane
 * x = nx-2 (every site counted, walls as zero); cl_set_flow_pressure is
 * NSdomainSetup's new deltaP (rho_in = 1, rho_out = 1 - 3 deltaP), followed by
 * cl_flow_init; cl_set_transport sets the solute relaxation frequencies and
 * the transport time step derived from the calibrated flow
 * (complab.cpp:708-727); the values of immobile solutes are not used (with a
 * zero diffusion coefficient their frequency is 2). */
int cl_flow_velocity_stats(cl_ctx* ctx, double* pore_mean_u, double* max_ux, double* outlet_mean_ux);
int cl_set_flow_pressure(cl_ctx* ctx, double rho_in, double rho_out);
/* The masked pore mean of the same calibration when a sessile microbe exists
 * (complab.cpp:625-640): the sum of the velocity norm and the number of sites
 * over the sites of material `code` in x = 1..nx-2 (MaskedScalarCounts3D and
 * the masked computeAverage(*computeVelocityNorm)); the caller weights the
 * pore and biofilm materials as the reference does. */
int cl_flow_velocity_norm_masked(cl_ctx* ctx, int32_t code, double* sum_norm, int64_t* count);
int cl_set_transport(cl_ctx* ctx, const double* omega_pore, const double* omega_bio, double dt);

/* ---- transport step ----------------------------------------------------------
 * cl_ade_init: initializeAtEquilibrium(c0, u=0) for every solute
 *              (src/complab_functions.hh:334-336).
 * cl_step:     n transport steps in the reference's order (src/complab.cpp:1252-1374,
 *              1849-1857): collide -> kinetics -> update_rxnLattices -> abiotic
 *              (+ dissolution) -> update_abiotic_rxnLattices -> equilibrium -> stream.
 *              Every step ends with geometry updates only when the caller asks
 *              (cl_precip_convert / cl_dissol_convert), as the reference gates them
 *              on an interval. */
int cl_ade_init(cl_ctx* ctx);
int cl_step(cl_ctx* ctx, int32_t n);

/* The step taken apart, for callers that keep the reference's processor
 * calls (src/complab.cpp:1252-1374, 1849-1857):
 *   cl_op_collide      collide of every mobile solute, populations written back
 *                      in place (AdvectionDiffusionBGKdynamics collide());
 *   cl_op_kinetics     run_kinetics + update_rxnLattices (part1.hh:63-146, 338-429);
 *   cl_op_surrogate    run_surrogate3D + update_rxnLattices (surrogate.hh:74-295);
 *   cl_op_abiotic      the dC reset, run_abiotic_kinetics or surfaceAbioticKinetics3D,
 *                      surfaceDissolutionKinetics3D, update_abiotic_rxnLattices
 *                      (part1.hh:158-336, precipitationVOP.hh:53-145,
 *                      dissolutionVOP.hh:265-435);
 *   cl_op_equilibrium  run_equilibrium_biotic (part4_eqsolver.hh:1355-1494);
 *   cl_op_reactions    the processors of the mask `ops` in one pass (kinetics and
 *                      surrogate then share one increment, as they share dC);
 *   cl_op_stream       stream (and the x-face boundary sites), ending the step.
 * cl_op_collide, any reaction operators, cl_op_stream is one cl_step (to FP32
 * rounding: the reactions read densities summed after the collision); the
 * reaction operators also run alone on the current state.  The node
 * conversions and the biofilm automaton are cl_precip_convert,
 * cl_dissol_convert and cl_ca_redistribute.  Each call synchronises; the
 * rate table only (a compiled rate law runs in cl_step). */
#define CL_OP_KINETICS    1
#define CL_OP_SURROGATE   2
#define CL_OP_ABIOTIC     4
#define CL_OP_EQUILIBRIUM 8
#define CL_OP_ALL         15
int cl_op_collide(cl_ctx* ctx);
int cl_op_kinetics(cl_ctx* ctx);
int cl_op_surrogate(cl_ctx* ctx);
int cl_op_abiotic(cl_ctx* ctx);
int cl_op_equilibrium(cl_ctx* ctx);
int cl_op_reactions(cl_ctx* ctx, int32_t ops);
int cl_op_stream(cl_ctx* ctx);

/* Compiled chemistries.  The reference compiles its rate laws into the
 * program (defineKinetics.hh / defineAbioticKinetics.hh, included by
 * src/complab.cpp); the library likewise compiles chemistries in, each a fixed
 * structure (solute and microbe counts, which solutes are mobile, the rate
 * laws' terms, the number of equilibrium components) whose values still come
 * from cl_config.  cl_create selects the compiled chemistry whose structure
 * the configuration has; its transport step runs in one launch with every
 * voxel's state in registers.  Other configurations run the run-time rate
 * table.  Both give the same fields.
 *   CL_OPT_COMPILED_CHEM  set: 0 = use the run-time table even when a compiled
 *                         chemistry matches, 1 = use it (default);
 *                         get: the id of the compiled chemistry in use, 0 = none. */
#define CL_OPT_COMPILED_CHEM 1
#define CL_OPT_FAST_VARIANT  2   /* launch shape of the compiled chemistry's step, 0..3 */
/* The learned warm start in the step (a compiled chemistry with Newton
 * speciation of 1..5 components; no counterpart in the reference).
 *   CL_OPT_EQ_LEARN  set K > 0: every step stores the (totals -> log10 free
 *                    components) pairs of a sampled one in 16 of the converged
 *                    voxels in a ring on the device (2^20 pairs); every K steps
 *                    the library's network (n_comp -> 64 -> 64 -> n_comp, GELU,
 *                    BF16 weights, FP32 accumulate) is trained on the device on
 *                    the ring (two epochs) and the ring is emptied.  Once
 *                    trained, a voxel with no previous solution of its own starts
 *                    Newton from the network's guess, with the reference's cold
 *                    start after eq.warm_iter iterations.  0: off.  get: K.
 *   CL_OPT_EQ_FORGET set: every voxel forgets its previous solutions (the next
 *                    step starts each solve from the network or cold).
 *   CL_OPT_EQ_LEARN_TRAININGS get: trainings done so far. */
#define CL_OPT_EQ_LEARN            3
#define CL_OPT_EQ_FORGET           4
#define CL_OPT_EQ_LEARN_TRAININGS  5
int cl_set_option(cl_ctx* ctx, int32_t key, int64_t value);
int cl_get_option(cl_ctx* ctx, int32_t key, int64_t* value);

/* field access (host FP64 buffers of nx*ny*nz values) */
#define CL_FIELD_CONC      0   /* solute density (index = solute) */
#define CL_FIELD_BIOMASS   1   /* sessile biomass (index = microbe) */
#define CL_FIELD_VELOCITY  2   /* coupled velocity component (index = 0,1,2) */
#define CL_FIELD_FLOW_RHO  3   /* flow density rho */
#define CL_FIELD_FLOW_U    4   /* flow velocity j computed from the populations (index = 0,1,2) */
#define CL_FIELD_PHASE     5   /* phase id */
#define CL_FIELD_EQ_ITERS  6   /* Newton iterations of the last equilibrium step */
int cl_get_field(cl_ctx* ctx, int32_t field, int32_t index, double* host_out);
int cl_set_field(cl_ctx* ctx, int32_t field, int32_t index, const double* host_in);

/* raw populations (debug/parity, checkpoints): flow 19*N floats as deviations
 * f-t_i in the natural (post-stream) order; solute s: 7*N floats of g_i.
 * Reading the flow needs a flow field (cl_flow_init or a set), setting it the
 * mask (CL_ERR_STATE otherwise); setting a solute's needs cl_ade_init.  A
 * get followed by a set restores the state bit for bit, at either parity. */
int cl_get_flow_populations(cl_ctx* ctx, float* host_out);
int cl_set_flow_populations(cl_ctx* ctx, const float* host_in);
int cl_get_solute_populations(cl_ctx* ctx, int32_t s, float* host_out);
int cl_set_solute_populations(cl_ctx* ctx, int32_t s, const float* host_in);

/* ---- measurement ----------------------------------------------------------------
 * CUDA events recorded on the context's stream around every launch of the
 * named kernel while timing is on; cl_timing_read synchronises and returns the
 * summed device time and the number of timed launches since the last read.
 * cl_launch_count: kernels this context launched since it was created. */
#define CL_KERNEL_ADE_MAIN  0   /* transport collide-stream of the interior sites (+ the reaction increments) */
#define CL_KERNEL_FLOW_STEP 1   /* D3Q19 collide-stream */
#define CL_KERNEL_ADE_REACT 2   /* the reaction chain of the reactive sites (kinetics .. equilibrium) */
int cl_timing_enable(cl_ctx* ctx, int32_t on);
int cl_timing_read(cl_ctx* ctx, int32_t kernel, double* total_ms, int64_t* launches);
int cl_launch_count(const cl_ctx* ctx, int64_t* launches);

/* network of the surrogate reaction type, slot 0..CL_MAX_SRG_ORG-1 (before cl_step) */
int cl_set_surrogate(cl_ctx* ctx, int32_t slot, const cl_surrogate_net* net);

/* ---- cellular-automaton biofilm -------------------------------------
 * One call is the CA block of the reference's step (src/complab.cpp:1453-1715):
 * updateLocalMaskNtotalLattices3D, then while the biomass maximum exceeds
 * ca_bmax: a push sweep (pushExcessBiomass3D / halfPushExcessBiomass3D,
 * complab3d_processors_part1.hh:432-894), the mask / total update, and every
 * 50 sweeps the age wavefront (updateAgeDistance3D, part2.hh:717-842) to a
 * fixed point.  The push sweep runs on every over-full voxel at once: the
 * totals that decide capacities are the sweep's starting values (as the
 * reference reads its total lattice, updated only between sweeps), each
 * voxel's outflows are gathered by its neighbours in a fixed order, and a
 * counter-based hash of (seed, sweep, site) replaces std::rand.  *sweeps =
 * push sweeps run, *mask_changes = sites whose mask changed; returns
 * CL_WARN_NOT_CONVERGED when 100 sweeps bring no decrease of the maximum,
 * when an age relaxation takes more than 1000 passes, or after 1001 sweeps
 * (the reference ends the run there), and CL_ERR_DIVERGED on a non-finite
 * biomass.  The ages start at cl_ade_init: -1 wall, 0 pore, 1 biofilm. */
int cl_ca_redistribute(cl_ctx* ctx, int32_t* sweeps, int64_t* mask_changes, double* bmax_after);
/* updateLocalMaskNtotalLattices3D alone: the initial mask update after the
 * biomass is seeded (complab.cpp:1068-1076).  It also resets the mask-sum
 * baseline: cl_ca_redistribute runs one age pass when the sum of the mask
 * has moved since the last baseline (complab.cpp:1736-1739).  cl_ade_init
 * sets the first baseline from the uploaded mask. */
int cl_ca_update_mask(cl_ctx* ctx, int64_t* mask_changes);
/* fdDiffusion3D (src/complab3d_processors_part2.hh:258-420), the
 * finite-difference biomass solver (solver_type FD): one explicit step
 * B += nu * laplacian(B) of the sessile biomass of the microbes whose bit is
 * set in `microbes`, on the sites of x = 1 .. nx-2 whose material number
 * exceeds 1, with no flux into sites whose material number is below 2 or
 * out of the lattice; nu in lattice units (the reference passes
 * bioNUinPore[0]).  The reference's step is cl_ca_update_mask, this, and
 * cl_ca_update_mask again (complab.cpp:1716-1731). */
int cl_fd_diffuse(cl_ctx* ctx, double nu, uint32_t microbes);
/* the age field (read) as FP64 */
#define CL_FIELD_CA_AGE    7
#define CL_FIELD_CA_TOTAL  8   /* total biomass the CA last computed */
/* the Newton warm starts of the transport step (eq_warm_previous), read and
 * written for checkpoints: index j < n_comp the last converged log10 free
 * component j of each site, n_comp <= j < 2 n_comp the one before; NaN where
 * a site has none (stored in FP32) */
#define CL_FIELD_EQ_START  9
/* the sites' dynamics (index 0 the flow's, 1 the solutes'): 0 NoDynamics,
 * 1 bounce-back, 2 pore, 3 biofilm.  They follow the mask at upload and then
 * change only by cl_update_dynamics, the reference's dynamics switches, so
 * after node conversions they are part of the state a checkpoint keeps
 * (a precipitated voxel keeps its solute dynamics, complab.cpp:1829-1836) */
#define CL_FIELD_DYNAMICS 10

/* ---- reductions ----------------------------------------------------- */
#define CL_RED_SUM   0
#define CL_RED_MIN   1
#define CL_RED_MAX   2
#define CL_RED_COUNT_EQ 3          /* count of sites whose mask == (int)arg */
int cl_reduce(cl_ctx* ctx, int32_t field, int32_t index, int32_t op, double arg, double* out);

/* ---- geometry updates --------------------------------------------
 * precipNodeConversion3D (src/precipitationVOP.hh:158-219; stamps
 * precip_phase_id on the voxels it seals) and dissolNodeConversion3D
 * (src/dissolutionVOP.hh:459-527; reopens to the first pore code).  *changed =
 * number of sites whose mask changed; the reaction gates follow the new mask at
 * once, the flow / solute dynamics only after cl_update_dynamics, as in the
 * reference's loop (complab.cpp:1783-1845).  Mineral release
 * (surfaceDissolutionKinetics3D, :265-435) runs inside cl_step when
 * dissol_enabled; the phase lattice is seeded from the mask by cl_upload_mask
 * (initPhaseLattice3D) and the grain inventories by cl_ade_init.
 * CL_FIELD_PHASE reads and writes the phase ids (0 = none). */
int cl_precip_convert(cl_ctx* ctx, int64_t* changed);
int cl_dissol_convert(cl_ctx* ctx, int64_t* changed);

/* ---- speciation batch ----------------------------------------------------------
 * One FP64 Newton solve per entry.  totals: n*n_comp component totals T_j.
 * logfree_io: n*n_comp log10 free component concentrations; on input the start
 *   used by CL_EQ_START_GIVEN, on output the solution.
 * iters: Newton iterations used (may be NULL).  status: 0 converged from the
 *   first start, 1 converged after the cold fallback, 2 not converged (may be NULL).
 * Residual: max_j |sum_i S_ij c_i - T_j| / sum_i |S_ij| c_i <= eq->tol. */
#define CL_EQ_START_COLD    0   /* reference rule: log10 of the component's own species, else 1e-7 */
#define CL_EQ_START_GIVEN   1   /* start from logfree_io */
#define CL_EQ_START_LEARNED 2   /* start from the context's trained network */
typedef struct cl_eq_solver cl_eq_solver;
cl_eq_solver* cl_eq_create(const cl_eq_system* sys, void* stream, int* status);
int cl_eq_destroy(cl_eq_solver* s);
/* device-pointer variant (inputs already in HBM) */
int cl_eq_solve_device(cl_eq_solver* s, const double* d_totals, const double* d_cold_species,
                       double* d_logfree, int32_t* d_iters, uint8_t* d_status,
                       int64_t n, int32_t start);
/* host-buffer variant (copies inside) */
int cl_eq_solve_host(cl_eq_solver* s, const double* totals, const double* cold_species,
                     double* logfree, int32_t* iters, uint8_t* status,
                     int64_t n, int32_t start);

/* Batch speciation that allocates nothing (no counterpart in the reference).
 * For callers that must not allocate device memory: code running under a
 * framework's caching allocator that owns the GPU's memory budget, and code
 * between the kernels of a stream-ordered sequence, where cudaMalloc/cudaFree
 * would synchronise the device.  Same solve as cl_eq_solve_device with start
 * CL_EQ_START_COLD or CL_EQ_START_GIVEN (warm start with cold fallback when
 * cold_species is given), on caller-owned device buffers and `stream`; no
 * solver object is needed.  The fallback list lives in a fixed array of
 * CL_EQ_NOALLOC_MAX_N entries (8 MiB) that every GPU loading the library
 * holds until exit; larger n is rejected with CL_ERR_ARG.  The first call on
 * a device looks up that array's device address, so make it before any
 * stream capture, and do not reset the device (cudaDeviceReset) between
 * calls: the address belongs to the context such a reset destroys.  All
 * calls share the array: calls that overlap on the GPU race, and it keeps the
 * last call's contents (the counter is cleared on every call). */
#define CL_EQ_NOALLOC_MAX_N       1048576
#define CL_EQ_NOALLOC_MAX_DEVICES 64
int cl_eq_solve_noalloc(const cl_eq_system* sys, const double* d_totals, const double* d_cold_species,
                        double* d_logfree, int32_t* d_iters, uint8_t* d_status,
                        int64_t n, int32_t start, void* stream);

/* The reference's live speciation entry point, calculate_species_concentrations
 * (src/complab3d_processors_part4_eqsolver.hh:1187-1214): per entry, the
 * component totals of the given species (clamped to [1e-30, 10]), the PCF +
 * Anderson solve from the reference's cold start, and the species it returns
 * (non-equilibrium species pass through clamped; NaN / inf fall back to the
 * input).  species_in / species_out: n*n_species.  iters: the reference's
 * iteration count (getLastIterations); converged: 1 if ||f||_2 < tol was
 * reached (didConverge).  Either may be NULL.  Uses the solver's tableau,
 * max_iter, tol and anderson_depth.  Returns CL_WARN_NOT_CONVERGED if some
 * entry did not converge. */
int cl_eq_pcf_device(cl_eq_solver* s, const double* d_species_in, double* d_species_out,
                     int32_t* d_iters, uint8_t* d_converged, int64_t n);
int cl_eq_pcf_host(cl_eq_solver* s, const double* species_in, double* species_out,
                   int32_t* iters, uint8_t* converged, int64_t n);

/* ---- learned warm start: MLP n_comp -> 64 -> 64 -> n_comp, GELU, BF16 weights,
 *      FP32 accumulate, trained on the device by the library's own forward and
 *      backward kernels on pairs (log10 T -> log10 free) that Newton produced. */
int cl_eq_train(cl_eq_solver* s, const double* d_totals, const double* d_logfree,
                int64_t n_pairs, int32_t epochs, int32_t batch, float lr, uint64_t seed,
                float* final_loss);
/* one forward+backward of a batch, for gradient checks: x n*n_comp inputs
 * (log10 T), y n*n_comp targets; writes the loss and the FP32 gradients in the
 * layout of cl_eq_get_params.  Host buffers. */
int cl_eq_grad_host(cl_eq_solver* s, const float* x, const float* y, int32_t n,
                    float* loss, float* grads);
#define CL_MLP_HIDDEN 64
int cl_eq_param_count(const cl_eq_solver* s, int32_t* count);
int cl_eq_get_params(cl_eq_solver* s, float* host_params);
int cl_eq_set_params(cl_eq_solver* s, const float* host_params);
int cl_eq_predict_host(cl_eq_solver* s, const float* x, float* y, int32_t n);
/* The tensor-core path of the network's inference (cl_eq_predict_*, the
 * learned start of cl_eq_solve_*): CL_EQ_NET_TCGEN05 (default) runs 128
 * samples per CTA through tcgen05.mma with the accumulators in tensor memory;
 * CL_EQ_NET_MMA_SYNC runs 64-sample tiles through warp-level mma.sync.  Both
 * take BF16 operands and activations with FP32 accumulation.  Training
 * (cl_eq_train, cl_eq_grad_host) runs the warp-level path.  A tcgen05
 * inference whose wait on its MMAs times out is reported as CL_ERR_CUDA by
 * cl_eq_predict_host. */
#define CL_EQ_NET_TCGEN05  0
#define CL_EQ_NET_MMA_SYNC 1
int cl_eq_set_network_path(cl_eq_solver* s, int32_t path);
/* the network's start for n device totals (log10 free components, FP64), the
 * values CL_EQ_START_LEARNED starts Newton from; no counterpart in the reference */
int cl_eq_predict_device(cl_eq_solver* s, const double* d_totals, double* d_logfree, int64_t n);

#define CL_SRG_TENSOR 0   /* BF16 tensor-core inference, FP32 accumulate */
#define CL_SRG_FP32   1   /* FP32 CUDA-core reference kernel */
#define CL_SRG_TCGEN05 2  /* BF16 on tcgen05.mma, FP32 accumulators in tensor memory (128 voxels per CTA);
                             cl_surrogate_batch_host reports a timed-out MMA wait as CL_ERR_CUDA */
int cl_surrogate_batch_device(const cl_surrogate_net* net, const float* d_x, float* d_y,
                              int64_t n, int32_t mode, void* stream);
int cl_surrogate_batch_host(const cl_surrogate_net* net, const float* x, float* y,
                            int64_t n, int32_t mode);

#ifdef __cplusplus
}
#endif
#endif /* COMPLAB_GPU_H */
