// internal.h -- context layout and kernel-launch declarations shared by the
// translation units of libcomplab_gpu.so.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
struct cl_eq_solver;
#include <cstdint>
#include <string>
#include <vector>
#include "../../include/complab_gpu.h"
#include "lattice.cuh"

namespace cl {

void set_error(const std::string& msg);
int  cuda_fail(cudaError_t e, const char* where);

#define CL_CUDA(call) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return ::cl::cuda_fail(e_, #call); } while (0)
#define CL_LAUNCH_CHECK(where) do { cudaError_t e_ = cudaGetLastError(); if (e_ != cudaSuccess) return ::cl::cuda_fail(e_, where); } while (0)

// Flow-convergence tracer state on the device (Palabos util::ValueTracer, window 500).
struct FlowTracer {
    double window[500];
    int    count, head;
    int    converged;      // 1 once stddev/avg < eps (or NaN)
    int    diverged;       // NaN ratio
    int    steps_done;     // steps executed since the tracer was armed
    int    converged_at;   // steps_done value when it converged
    double last_energy;
    double eps;
};

// A surrogate network as the transport kernel reads it: FP32 parameters in
// device memory (W then b, layer by layer) and the mapminmax settings.
struct SrgNetDev {
    int L;
    int w[CL_SRG_MAX_LAYERS + 1];
    int poff[CL_SRG_MAX_LAYERS];
    float xo[CL_SRG_MAX_WIDTH], xg[CL_SRG_MAX_WIDTH], xlo[CL_SRG_MAX_WIDTH], xhi[CL_SRG_MAX_WIDTH];
    float yo[CL_SRG_MAX_WIDTH], yg[CL_SRG_MAX_WIDTH];
    float xymin, yymin;
    const float* params;
};

// The equilibrium settings the transport kernels read (the tableau itself
// travels as EqDev).
struct EqParams {
    int    n_comp, n_species;
    int    max_iter, warm_iter, solver, anderson_depth;
    double tol;
};

// Per-solute transport parameters passed by value to the transport kernels.
struct AdeParams {
    int    S;                          // all solutes
    int    n_mob;                      // mobile solutes
    int    mob_index[CL_MAX_SOLUTES];  // solute index of mobile slot k
    int    mob_slot[CL_MAX_SOLUTES];   // mobile slot of solute s, or -1 if immobile
    float  omega_pore[CL_MAX_SOLUTES]; // per mobile slot
    float  omega_bio[CL_MAX_SOLUTES];
    int    left_neu[CL_MAX_SOLUTES], right_neu[CL_MAX_SOLUTES];   // per mobile slot
    float  left_val[CL_MAX_SOLUTES], right_val[CL_MAX_SOLUTES];
    int    M;                          // microbes
    double dt;
    int    do_kin, do_abio, surface_only, do_eq, eq_warm;
    int    n_rxn;
    cl_rxn rxn[CL_MAX_RXN];
    double decay[CL_MAX_MICROBES];
    int    carrier[CL_MAX_MICROBES];   // solute whose density is microbe m's biomass, or -1 (sessile)
    int    n_carried;
    EqParams eq;
    int    solid_code, bb_code;
    int    n_srg;
    cl_srg_organism srg[CL_MAX_SRG_ORG];
    SrgNetDev net[CL_MAX_SRG_ORG];
    // dissolution: phase id k+1 is phase[k] (ids are checked to be 1..n_phases)
    int    do_dissol, dissol_surface_only, dissol_walls, n_phases;
    cl_phase phase[CL_MAX_PHASES];
};

// What a captured run of flow steps depends on: the launches it replays
// read these, so a graph is reused only while all of them are unchanged.
struct FlowGraphKey {
    const void* f; const void* list; const void* sidx; const void* cls; const void* tracer; const void* part;
    int64_t count, n_bgk;
    double tau_ns, perm_ratio, rho_in, rho_out;
    int energy_blocks, nodyn_coupled, use_tracer, parity;
    cudaStream_t stream;
};

struct Ctx {
    cl_config cfg;
    Geo geo;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool mask_ready = false, flow_ready = false, ade_ready = false;
    // geometry
    uint8_t* d_mask = nullptr;       // material numbers
    uint8_t* d_ns_cls = nullptr;     // flow node class
    uint8_t* d_ade_cls = nullptr;    // transport node class | F_REACTIVE | F_SURFACE
    int64_t  n_bgk = 0;              // flow BGK sites (energy average denominator)
    bool     flow_nodyn_coupled = true;   // some NoDynamics site touches a flow site
    bool     ade_nodyn_coupled = true;
    // flow
    float*   d_f = nullptr;          // 19*N deviations
    int      flow_parity = 0;        // steps done mod 2
    double*  d_energy_part = nullptr;
    int      energy_blocks = 0;
    FlowTracer* d_tracer = nullptr;
    // transport
    AdeParams ap;
    float*   d_g = nullptr;          // n_mob*7*N
    int      ade_parity = 0;
    double*  d_imm = nullptr;        // S*N (only immobile slots used)
    double*  d_bio = nullptr;        // M*N
    float*   d_u = nullptr;          // 3*N
    float*   d_rho_adj = nullptr;    // n_mob*2*plane : pre-collision density next to each x face
    int32_t* d_eq_iters = nullptr;   // N
    float*   d_srg_params[CL_MAX_SRG_ORG] = {nullptr, nullptr};
    std::vector<float> h_srg_params[CL_MAX_SRG_ORG];   // host copies (a compiled chemistry's kernel takes them)
    double*  d_fd_copy = nullptr;        // the sessile biomass before a finite-difference step
    cudaGraphExec_t flow_graph = nullptr;   // a captured run of flow steps, valid for flow_graph_key
    FlowGraphKey flow_graph_key{};
    float*   d_eq_x = nullptr;       // n_comp*N previous converged log10 free components, by storage index (NaN: none)
    float*   d_eq_xp = nullptr;      // n_comp*N the solution before that, by storage index (NaN: none)
    uint8_t* d_phase = nullptr;      // N dissolvable phase id, 0 = none (dissolution only)
    double*  d_ca_total = nullptr;   // N total biomass (cellular automaton)
    int32_t* d_ca_age = nullptr;     // 2*N age wavefront, ping-pong
    uint8_t* d_ca_distpos = nullptr; // N: the reference's distance field is positive (non-wall, not on a last index)
    double*  d_ca_out = nullptr;     // 6*M*N outflow of each voxel per face and microbe in one sweep
    uint64_t ca_sweeps = 0;          // sweeps run so far (the generator's counter)
    int      ca_age_src = 0;         // age plane holding the current ages
    int64_t  ca_mask_sum = -1;       // mask sum at the last check (complab.cpp old_totMask)
    double*  d_rel = nullptr;        // S*N this step's release of each phase voxel: products per open
                                     // face, and at the phase substrate the voxel's own decrement
    // transport slots are stored compactly: site n's populations live at
    // storage index sidx[n] (stride N per population array); -1 = never needed
    // so far, its slots still hold the initial values
    int32_t* d_sidx = nullptr;       // N
    uint32_t* d_site_of = nullptr;   // N capacity: site of each storage index
    int64_t  n_stored = 0;
    bool     store_dirty = true;     // classes changed: the needed set may have grown
    // flow slots are stored the same way: the sites that stream and their 18
    // D3Q19 neighbours; an unstored site's slots hold 0 (flow_init gives every
    // non-BGK site 0, and BGK sites always stream)
    int32_t* d_fsidx = nullptr;      // N
    int64_t  n_fstored = 0;
    bool     fstore_dirty = true;
    float*   d_dc = nullptr;         // n_mob*N this step's reaction increment of each reactive site, by storage
                                     // index (dense for a warp's run of live sites, like the populations)
    uint32_t* d_live = nullptr;      // the live interior sites of the transport, increasing (live list)
    uint32_t* d_flive = nullptr;     // the flow's sites that stream, increasing
    int64_t  n_flive = 0;
    bool     flive_dirty = true;
    int64_t  n_live = 0;
    bool     live_dirty = true;     // classes changed since the list was built
    int64_t* d_live_blk = nullptr;  // per-block counts / offsets of the list build
    // the step's slabs of x planes: the reaction launch of slab j+1 (stream
    // s_react) runs while slab j streams (s_stream)
    static constexpr int kMaxSlabs = 64;
    int      slabs = 1;
    int64_t  slab_site[kMaxSlabs + 1] = {};    // first site of each slab (interior x)
    int64_t  slab_live[kMaxSlabs + 1] = {};   // first live-list entry of each slab
    cudaStream_t s_react = nullptr, s_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_slab[kMaxSlabs] = {};
    unsigned long long* d_counters = nullptr;  // [0] non-converged Newton solves, [1] transport / [2] flow sites without storage
    // scratch for reductions / field IO
    double*  d_scratch = nullptr;
    size_t   scratch_bytes = 0;
    uint64_t device_bytes = 0;
    // measurement: event pairs around timed kernels, launch counter
    static constexpr int kTimedKernels = 3, kEventPool = 512;
    bool     timing = false;
    cudaEvent_t ev[kTimedKernels][kEventPool][2] = {};
    int      ev_used[kTimedKernels] = {0, 0, 0};
    double   ev_ms[kTimedKernels] = {0.0, 0.0, 0.0};
    int64_t  ev_launches[kTimedKernels] = {0, 0, 0};
    int64_t  launches = 0;
    // compiled chemistry (chem.cuh) whose structure this configuration has,
    // 0 = none; its one-launch transport step runs while chem_on
    int      chem = 0;
    bool     chem_on = true;
    int      fast_variant = 0;   // launch shape of the one-launch step (block size, blocks per SM)
    // learned warm start inside the step (learned.cuh): the network and its
    // trainer, the ring of sampled converged pairs, the training interval
    cl_eq_solver* learn = nullptr;
    int      learn_interval = 0;        // steps between trainings, 0 = off
    int      learn_shift = 4;           // one converged voxel in 2^shift joins the ring per step
    int      learn_epochs = 2;
    bool     learn_ready = false;       // the network has been trained at least once
    double*  d_pair_T = nullptr;        // [cap][n_comp]
    double*  d_pair_X = nullptr;
    unsigned long long* d_pair_count = nullptr;
    int64_t  pair_cap = 0;
    int64_t  learn_steps = 0;           // steps since the last training
    int64_t  step_index = 0;            // steps taken (the ring's sample salt)
    float    learn_loss = 0.f;
    int64_t  learn_trainings = 0;
    bool     op_collided = false;       // cl_op_collide ran; cl_op_stream completes the step
};

// the network of a speciation solver for the step's learned start: FP32
// master weights and standardisation (device), trained flag
int eq_solver_network(cl_eq_solver* s, const float** master, const float** norm, int* trained);

// event bracket around one launch of a timed kernel (no-op when timing is off)
int timing_begin(Ctx* c, int kernel);
int timing_end(Ctx* c, int kernel);

// kernels (launchers return a CL_* status)
int flow_init(Ctx* c);
int flow_step(Ctx* c, int arm_tracer_flag);
int flow_arm_tracer(Ctx* c, double eps);
int flow_macro(Ctx* c, double* d_rho, float* d_u3, int want_bc_velocity);
int flow_stats(Ctx* c, double out[3]);
int flow_norm_masked(Ctx* c, int code, double out[2]);   // sum |u| and count of one material, x = 1..nx-2   // sum |u| and max u_x over x = 1..nx-2, sum u_x at x = nx-2
int classes_from_mask(Ctx* c);
int ade_init(Ctx* c);
int ade_step(Ctx* c);
int ade_step_fast(Ctx* c);
// the per-operator entry points (ops.cu)
int ops_collide(Ctx* c);
int ops_react(Ctx* c, int ops);
int ops_stream(Ctx* c);      // the transport step of the compiled chemistry c->chem
int fd_diffuse(Ctx* c, double nu, uint32_t sel);   // fdDiffusion3D of the microbes in sel
int chem_match(const cl_config& cfg);   // id of the compiled chemistry cfg has the structure of, or 0
bool chem_ready(const Ctx* c);          // the context holds what its compiled chemistry needs
const char* chem_name(int id);
int ade_density(Ctx* c, int s, double* d_out);
int flow_population_io(Ctx* c, float* d_natural, int to_natural);
int ade_population_io(Ctx* c, int slot, float* d_natural);
int precip_convert(Ctx* c, int64_t* changed);
int dissol_convert(Ctx* c, int64_t* changed);
int phase_seed(Ctx* c);          // grain phases from the mask (initPhaseLattice3D)
int phase_fill(Ctx* c);          // grain inventories (initial_fill) after ade_init
int refresh_flags(Ctx* c);       // class flags after a mask / phase change, dynamics kept
int build_live_list(Ctx* c);    // the live interior sites of the transport classes, in site order
int build_flow_list(Ctx* c);    // the flow sites that stream (not bounce-back), in site order
// store the sites the transport now needs (all: every site; extra: a device
// byte per site, nonzero where a site must be stored as well)
int store_update(Ctx* c, int all, const uint8_t* extra = nullptr);
int ade_population_set(Ctx* c, int slot, const float* d_nat);   // natural order -> storage
int eq_start_io(Ctx* c, int j, double* d_nat, int to_natural);   // Newton warm start j <-> natural order
// storage indices for the sites flagged in need, after the *n_stored assigned
int assign_storage(Ctx* c, const uint8_t* need, int32_t* sidx, uint32_t* site_of, int64_t* n_stored,
                   int64_t* first, int64_t* added);
int flow_store_update(Ctx* c, const float* d_natural);  // store the sites the flow needs (+ nonzero inputs)
int ca_init(Ctx* c);             // ages and the distance sign from the mask
int ca_redistribute(Ctx* c, int32_t* sweeps, int64_t* mask_changes, double* bmax_after);
int ca_update_mask(Ctx* c, int64_t* mask_changes);
int ca_field(Ctx* c, int which, double* d_out);   // CL_FIELD_CA_AGE / CL_FIELD_CA_TOTAL into N doubles
int update_dynamics(Ctx* c);
int reduce_field(Ctx* c, const double* d_field, int op, double arg, const uint8_t* d_mask, double* out);

// alloc helper with accounting
template <typename T>
inline int dalloc(Ctx* c, T** p, size_t count) {
    size_t bytes = count * sizeof(T);
    if (bytes == 0) { *p = nullptr; return CL_OK; }
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) { *p = nullptr; return cuda_fail(e, "cudaMalloc"); }
    c->device_bytes += bytes;
    return CL_OK;
}

inline int grid_for(int64_t work, int block, int max_blocks) {
    int64_t b = (work + block - 1) / block;
    if (b > max_blocks) b = max_blocks;
    if (b < 1) b = 1;
    return (int)b;
}

}  // namespace cl
