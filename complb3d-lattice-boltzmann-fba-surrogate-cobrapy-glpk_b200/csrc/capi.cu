// capi.cu -- the C ABI of include/complab_gpu.h over the device context.
#include "internal.h"
#include <cstring>
#include <cstdlib>
#include <cstdio>
#include <vector>
#include <algorithm>
#include <cmath>

namespace cl {

static thread_local std::string g_err;
void set_error(const std::string& msg) { g_err = msg; }

// sum the elapsed time of the recorded pairs of one kernel and free the pool
static int fold_events(Ctx* c, int k) {
    for (int i = 0; i < c->ev_used[k]; ++i) {
        float ms = 0.f;
        cudaError_t e = cudaEventSynchronize(c->ev[k][i][1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, c->ev[k][i][0], c->ev[k][i][1]);
        if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
        c->ev_ms[k] += ms;
        c->ev_launches[k] += 1;
    }
    c->ev_used[k] = 0;
    return CL_OK;
}

int timing_begin(Ctx* c, int k) {
    if (!c->timing) return CL_OK;
    if (c->ev_used[k] == Ctx::kEventPool) { int r = fold_events(c, k); if (r) return r; }
    CL_CUDA(cudaEventRecord(c->ev[k][c->ev_used[k]][0], c->stream));
    return CL_OK;
}

// k >= 0: close the pair opened by timing_begin; k < 0: fold kernel -1-k
int timing_end(Ctx* c, int k) {
    if (k < 0) return fold_events(c, -1 - k);
    if (!c->timing) return CL_OK;
    CL_CUDA(cudaEventRecord(c->ev[k][c->ev_used[k]][1], c->stream));
    c->ev_used[k] += 1;
    return CL_OK;
}
int cuda_fail(cudaError_t e, const char* where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? CL_ERR_NOMEM : CL_ERR_CUDA;
}

static int validate(const cl_config* c) {
    if (!c) { set_error("null config"); return CL_ERR_ARG; }
    if (c->nx < 3 || c->ny < 1 || c->nz < 1) { set_error("lattice needs nx >= 3, ny >= 1, nz >= 1"); return CL_ERR_ARG; }
    if (c->n_solutes < 0 || c->n_solutes > CL_MAX_SOLUTES) { set_error("n_solutes out of range"); return CL_ERR_ARG; }
    if (c->n_microbes < 0 || c->n_microbes > CL_MAX_MICROBES) { set_error("n_microbes out of range"); return CL_ERR_ARG; }
    if (c->n_rxn < 0 || c->n_rxn > CL_MAX_RXN) { set_error("n_rxn out of range"); return CL_ERR_ARG; }
    if (c->rate_law != CL_RATELAW_TABLE && c->rate_law != CL_RATELAW_ZHAO) { set_error("unknown rate_law"); return CL_ERR_ARG; }
    for (int m = 0; m < CL_MAX_MICROBES; ++m) {
        const int cs = c->microbe_carrier[m];
        if (cs == 0) continue;
        if (m >= c->n_microbes || cs < 0 || cs > c->n_solutes || c->immobile[cs - 1]) {
            set_error("microbe_carrier must name a mobile solute (index + 1) of an existing microbe");
            return CL_ERR_ARG;
        }
        if (c->rate_law != CL_RATELAW_TABLE || c->n_srg > 0 || (c->ca_enabled && c->microbe_code[m] > 0)) {
            set_error("a microbe carried by a solute runs the rate table only (no surrogate, no CA on it)");
            return CL_ERR_ARG;
        }
    }
    {
        const int64_t N = (int64_t)c->nx * c->ny * c->nz;
        if (N * 19 >= (int64_t)1 << 32) { set_error("lattice too large: 19*nx*ny*nz must stay below 2^32"); return CL_ERR_ARG; }
    }
    if (c->n_pore_codes < 0 || c->n_pore_codes > CL_MAX_CODES || c->n_bio_codes < 0 || c->n_bio_codes > CL_MAX_CODES) {
        set_error("material code lists out of range"); return CL_ERR_ARG;
    }
    if (!(c->tau_ns > 0.5)) { set_error("tau_ns must exceed 0.5"); return CL_ERR_ARG; }
    for (int k = 0; k < c->n_rxn; ++k) {
        const cl_rxn& r = c->rxn[k];
        if (r.microbe >= c->n_microbes || r.n_monod < 0 || r.n_monod > CL_MAX_MONOD || r.n_mass < 0 || r.n_mass > 2) {
            set_error("rate table entry out of range"); return CL_ERR_ARG;
        }
        for (int j = 0; j < r.n_monod; ++j) if (r.monod_s[j] < 0 || r.monod_s[j] >= c->n_solutes) { set_error("monod solute index"); return CL_ERR_ARG; }
        for (int j = 0; j < r.n_mass; ++j) if (r.mass_s[j] < 0 || r.mass_s[j] >= c->n_solutes) { set_error("mass-action solute index"); return CL_ERR_ARG; }
    }
    if (c->n_srg < 0 || c->n_srg > CL_MAX_SRG_ORG) { set_error("n_srg out of range"); return CL_ERR_ARG; }
    for (int o = 0; o < c->n_srg; ++o) {
        const cl_srg_organism& g = c->srg[o];
        if (g.microbe < 0 || g.microbe >= c->n_microbes || g.net < 0 || g.net >= CL_MAX_SRG_ORG) {
            set_error("surrogate organism: microbe or network slot out of range"); return CL_ERR_ARG;
        }
        for (int i = 0; i < CL_SRG_MAX_WIDTH; ++i) {
            if ((g.in_kind[i] == CL_SRG_IN_FIN || g.in_kind[i] == CL_SRG_IN_CONC) &&
                (g.in_index[i] < 0 || g.in_index[i] >= c->n_solutes)) { set_error("surrogate input index"); return CL_ERR_ARG; }
            if (g.out_kind[i] == CL_SRG_OUT_FOUT && (g.out_index[i] < 0 || g.out_index[i] >= c->n_solutes)) {
                set_error("surrogate output index"); return CL_ERR_ARG;
            }
        }
    }
    if (c->n_phases < 0 || c->n_phases > CL_MAX_PHASES) { set_error("n_phases out of range"); return CL_ERR_ARG; }
    if (c->ca_enabled) {
        // complab_functions.hh:1167-1186: Bmax and the biofilm fraction are
        // required for a CA microbe; each microbe's biofilm material is its code
        if (c->n_microbes < 1) { set_error("the cellular automaton needs at least one microbe"); return CL_ERR_ARG; }
        if (!(c->ca_bmax > 0.0) || !std::isfinite(c->ca_bmax)) { set_error("ca_bmax must be positive"); return CL_ERR_ARG; }
        if (!(c->ca_thrd_frac >= 0.0) || !std::isfinite(c->ca_thrd_frac)) { set_error("ca_thrd_frac must be >= 0"); return CL_ERR_ARG; }
        if (c->n_pore_codes < 1) { set_error("the cellular automaton needs a pore material"); return CL_ERR_ARG; }
        for (int m = 0; m < c->n_microbes; ++m)
            if (c->microbe_code[m] < 0 || c->microbe_code[m] > 255) { set_error("microbe_code must be a material number 0..255"); return CL_ERR_ARG; }
    }
    if (c->dissol_enabled) {
        // complab.cpp:336-368: at least one phase, reopen_fraction in (0,1),
        // a substrate and a positive full density per phase
        if (c->n_phases < 1) { set_error("dissolution is enabled but no phase is declared"); return CL_ERR_ARG; }
        if (!(c->reopen_fraction > 0.0) || c->reopen_fraction >= 1.0) {
            set_error("reopen_fraction must lie in (0, 1)"); return CL_ERR_ARG;
        }
        for (int k = 0; k < c->n_phases; ++k) {
            const cl_phase& ph = c->phases[k];
            if (ph.id != k + 1) { set_error("phase ids must be 1..n_phases in declaration order"); return CL_ERR_ARG; }
            if (ph.substrate < 0 || ph.substrate >= c->n_solutes || !c->immobile[ph.substrate]) {
                set_error("a phase needs an immobile substrate for its inventory"); return CL_ERR_ARG;
            }
            if (!(ph.full_density > 0.0)) { set_error("phase full_density must be positive"); return CL_ERR_ARG; }
            if (ph.n_mass < 0 || ph.n_mass > 2) { set_error("phase rate law: 0..2 mass-action solutes"); return CL_ERR_ARG; }
            for (int j = 0; j < ph.n_mass; ++j)
                if (ph.mass_s[j] < 0 || ph.mass_s[j] >= c->n_solutes) { set_error("phase rate law solute index"); return CL_ERR_ARG; }
        }
        if (c->precip_phase_id < 0 || c->precip_phase_id > c->n_phases) { set_error("precip_phase_id out of range"); return CL_ERR_ARG; }
    }
    if (c->use_equilibrium) {
        const cl_eq_system& e = c->eq;
        if (e.n_comp < 1 || e.n_comp > 5 || e.n_species != c->n_solutes) {
            set_error("equilibrium in the transport step needs 1..5 components and one species per solute");
            return CL_ERR_ARG;
        }
        if ((e.solver != CL_EQ_SOLVER_NEWTON && e.solver != CL_EQ_SOLVER_PCF) || e.anderson_depth < 0 ||
            e.anderson_depth > 8) {
            set_error("unknown equilibrium solver, or anderson_depth outside 0..8");
            return CL_ERR_ARG;
        }
    }
    return CL_OK;
}

}  // namespace cl

using namespace cl;

struct cl_ctx { Ctx c; };

extern "C" {

const char* cl_last_error(void) { return g_err.c_str(); }

int cl_abi_sizes(int32_t* sizes, int32_t n) {
    const int32_t v[5] = {(int32_t)sizeof(cl_config), (int32_t)sizeof(cl_rxn), (int32_t)sizeof(cl_eq_system),
                          (int32_t)sizeof(cl_phase), (int32_t)sizeof(cl_surrogate_net)};
    int k = 0;
    for (; k < n && k < 5; ++k) sizes[k] = v[k];
    return k;
}

cl_ctx* cl_create(const cl_config* cfg, void* stream, int* status) {
    int st = validate(cfg);
    if (st != CL_OK) { if (status) *status = st; return nullptr; }
    cl_ctx* h = new cl_ctx();
    Ctx* c = &h->c;
    c->cfg = *cfg;
    c->geo.nx = cfg->nx; c->geo.ny = cfg->ny; c->geo.nz = cfg->nz;
    c->geo.plane = (int64_t)cfg->ny * cfg->nz;
    c->geo.N = c->geo.plane * cfg->nx;
    c->geo.by_nz.init((uint32_t)cfg->nz);
    c->geo.by_ny.init((uint32_t)cfg->ny);
    const int64_t N = c->geo.N;
    auto fail = [&](int s) { if (status) *status = s; cl_destroy(h); return (cl_ctx*)nullptr; };
    if (stream) { c->stream = (cudaStream_t)stream; c->own_stream = false; }
    else {
        cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
        c->own_stream = true;
    }
    {
        // the slab pipeline of the transport step: two streams and their events
        cudaError_t e = cudaStreamCreateWithFlags(&c->s_react, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->s_stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
        for (int j = 0; j < Ctx::kMaxSlabs && e == cudaSuccess; ++j)
            e = cudaEventCreateWithFlags(&c->ev_slab[j], cudaEventDisableTiming);
        if (e != cudaSuccess) return fail(cuda_fail(e, "slab streams"));
        // eight slabs of at least 32 planes each; small lattices run unsliced
        c->slabs = std::max(1, std::min(8, (cfg->nx - 2) / 32));
    }
    // transport parameters
    AdeParams& p = c->ap;
    std::memset(&p, 0, sizeof p);
    p.S = cfg->n_solutes;
    p.n_mob = 0;
    for (int s = 0; s < CL_MAX_SOLUTES; ++s) p.mob_slot[s] = -1;
    for (int s = 0; s < cfg->n_solutes; ++s) {
        if (cfg->immobile[s]) continue;
        const int m = p.n_mob++;
        p.mob_index[m] = s;
        p.mob_slot[s] = m;
        p.omega_pore[m] = (float)cfg->omega_pore[s];
        p.omega_bio[m] = (float)cfg->omega_bio[s];
        p.left_neu[m] = cfg->left_type[s] == CL_BC_NEUMANN;
        p.right_neu[m] = cfg->right_type[s] == CL_BC_NEUMANN;
        p.left_val[m] = (float)cfg->left_value[s];
        p.right_val[m] = (float)cfg->right_value[s];
    }
    p.M = cfg->n_microbes;
    p.dt = cfg->dt;
    int n_bio = 0, n_abio = 0;
    for (int k = 0; k < cfg->n_rxn; ++k) (cfg->rxn[k].microbe >= 0 ? n_bio : n_abio)++;
    p.do_kin = cfg->enable_kinetics && (n_bio > 0 || cfg->n_microbes > 0);
    p.do_abio = cfg->enable_abiotic && (n_abio > 0 || cfg->rate_law != CL_RATELAW_TABLE) && cfg->n_solutes > 0;
    p.surface_only = cfg->precip_enabled && cfg->abiotic_surface_only;
    p.do_eq = cfg->use_equilibrium;
    p.eq_warm = cfg->use_equilibrium && cfg->eq_warm_previous;
    p.n_rxn = cfg->n_rxn;
    for (int k = 0; k < cfg->n_rxn; ++k) p.rxn[k] = cfg->rxn[k];
    for (int m = 0; m < CL_MAX_MICROBES; ++m) p.decay[m] = cfg->decay[m];
    p.n_carried = 0;
    for (int m = 0; m < CL_MAX_MICROBES; ++m) {
        p.carrier[m] = m < cfg->n_microbes ? cfg->microbe_carrier[m] - 1 : -1;
        if (p.carrier[m] >= 0) ++p.n_carried;
    }
    p.eq.n_comp = cfg->eq.n_comp;
    p.eq.n_species = cfg->eq.n_species;
    p.eq.max_iter = cfg->eq.max_iter;
    p.eq.warm_iter = cfg->eq.warm_iter;
    p.eq.solver = cfg->eq.solver;
    p.eq.anderson_depth = cfg->eq.anderson_depth;
    p.eq.tol = cfg->eq.tol;
    p.solid_code = cfg->solid_code;
    p.bb_code = cfg->bb_code;
    p.n_srg = cfg->n_srg;
    for (int o = 0; o < CL_MAX_SRG_ORG; ++o) { p.srg[o] = cfg->srg[o]; p.net[o] = SrgNetDev{}; }
    p.do_dissol = cfg->dissol_enabled && cfg->n_phases > 0;
    p.dissol_surface_only = cfg->dissol_surface_only;
    p.dissol_walls = cfg->dissol_apply_at_walls;
    p.n_phases = cfg->n_phases;
    for (int k = 0; k < cfg->n_phases; ++k) p.phase[k] = cfg->phases[k];
    c->chem = chem_match(*cfg);
    if (cfg->rate_law != CL_RATELAW_TABLE && c->chem == 0) {
        set_error("the compiled rate law needs the layout it was written for (CL_RATELAW_ZHAO: 24 substrates "
                  "with 2, 4, 5, 6, 9, 13, 21, 22, 23 immobile, 12 microbes, no equilibrium, no dissolution)");
        return fail(CL_ERR_ARG);
    }
    // device memory
    int r = CL_OK;
    if ((r = dalloc(c, &c->d_mask, N)) || (r = dalloc(c, &c->d_ns_cls, N)) || (r = dalloc(c, &c->d_ade_cls, N)) ||
        (r = dalloc(c, &c->d_f, 19 * N)) || (r = dalloc(c, &c->d_u, 3 * N)) ||
        (r = dalloc(c, &c->d_g, (size_t)p.n_mob * 7 * N)) ||
        (r = dalloc(c, &c->d_imm, (size_t)(p.S - p.n_mob > 0 ? p.S : 0) * N)) ||
        (r = dalloc(c, &c->d_bio, (size_t)p.M * N)) ||
        (r = dalloc(c, &c->d_rho_adj, (size_t)p.n_mob * 2 * c->geo.plane)) ||
        (r = dalloc(c, &c->d_eq_iters, (size_t)(cfg->use_equilibrium ? N : 0))) ||
        (r = dalloc(c, &c->d_eq_x, (size_t)(p.eq_warm ? cfg->eq.n_comp : 0) * N)) ||
        (r = dalloc(c, &c->d_eq_xp, (size_t)(p.eq_warm ? cfg->eq.n_comp : 0) * N)) ||
        (r = dalloc(c, &c->d_phase, (size_t)(p.do_dissol ? N : 0))) ||
        (r = dalloc(c, &c->d_rel, (size_t)(p.do_dissol ? p.S : 0) * N)) ||
        (r = dalloc(c, &c->d_dc, (size_t)((p.do_kin || p.do_abio || p.n_srg > 0 || p.do_dissol ||
                                             cfg->use_equilibrium) ? p.n_mob : 0) * N)) ||
        (r = dalloc(c, &c->d_ca_total, (size_t)(cfg->ca_enabled ? N : 0))) ||
        (r = dalloc(c, &c->d_ca_age, (size_t)(cfg->ca_enabled ? 2 * N : 0))) ||
        (r = dalloc(c, &c->d_ca_distpos, (size_t)(cfg->ca_enabled ? N : 0))) ||
        (r = dalloc(c, &c->d_ca_out, (size_t)(cfg->ca_enabled ? 6 * p.M : 0) * N)) ||
        (r = dalloc(c, &c->d_counters, 8)) || (r = dalloc(c, &c->d_tracer, 1)))
        return fail(r);
    if (c->d_eq_x) cudaMemsetAsync(c->d_eq_x, 0xff, sizeof(float) * cfg->eq.n_comp * N, c->stream);  // NaN
    if (c->d_eq_xp) cudaMemsetAsync(c->d_eq_xp, 0xff, sizeof(float) * cfg->eq.n_comp * N, c->stream);
    c->energy_blocks = grid_for(N, 256, 148 * 8);
    if ((r = dalloc(c, &c->d_energy_part, c->energy_blocks))) return fail(r);
    c->scratch_bytes = sizeof(double) * ((size_t)N + 65536);
    if ((r = dalloc(c, &c->d_scratch, c->scratch_bytes / sizeof(double)))) return fail(r);
    cudaMemsetAsync(c->d_u, 0, sizeof(float) * 3 * N, c->stream);
    if (c->d_bio) cudaMemsetAsync(c->d_bio, 0, sizeof(double) * p.M * N, c->stream);
    cudaMemsetAsync(c->d_counters, 0, 8 * sizeof(unsigned long long), c->stream);
    if (c->d_eq_iters) cudaMemsetAsync(c->d_eq_iters, 0, sizeof(int32_t) * N, c->stream);
    if (c->d_phase) cudaMemsetAsync(c->d_phase, 0, N, c->stream);
    if (c->d_rel) cudaMemsetAsync(c->d_rel, 0, sizeof(double) * p.S * N, c->stream);
    cudaError_t e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cl_create"));
    if (status) *status = CL_OK;
    return h;
}

int cl_destroy(cl_ctx* h) {
    if (!h) return CL_OK;
    Ctx* c = &h->c;
    if (c->stream) cudaStreamSynchronize(c->stream);
    void* ptrs[] = {c->d_mask, c->d_ns_cls, c->d_ade_cls, c->d_f, c->d_u, c->d_g, c->d_imm, c->d_bio,
                    c->d_rho_adj, c->d_eq_iters, c->d_eq_x, c->d_eq_xp, c->d_phase, c->d_rel, c->d_counters, c->d_tracer,
                    c->d_energy_part, c->d_scratch, c->d_ca_total, c->d_ca_age, c->d_ca_distpos, c->d_ca_out,
                    c->d_dc, c->d_live, c->d_live_blk, c->d_sidx, c->d_site_of, c->d_flive, c->d_fsidx,
                    c->d_pair_T, c->d_pair_X, c->d_pair_count, c->d_fd_copy};
    if (c->learn) cl_eq_destroy(c->learn);
    if (c->flow_graph) cudaGraphExecDestroy(c->flow_graph);
    for (void* p : ptrs) if (p) cudaFree(p);
    for (int o = 0; o < CL_MAX_SRG_ORG; ++o) if (c->d_srg_params[o]) cudaFree(c->d_srg_params[o]);
    for (int k = 0; k < Ctx::kTimedKernels; ++k)
        for (int i = 0; i < Ctx::kEventPool; ++i)
            for (int j = 0; j < 2; ++j) if (c->ev[k][i][j]) cudaEventDestroy(c->ev[k][i][j]);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->s_react) cudaStreamDestroy(c->s_react);
    if (c->s_stream) cudaStreamDestroy(c->s_stream);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    for (int j = 0; j < Ctx::kMaxSlabs; ++j) if (c->ev_slab[j]) cudaEventDestroy(c->ev_slab[j]);
    delete h;
    return CL_OK;
}

int cl_device_bytes(const cl_ctx* h, uint64_t* bytes) {
    if (!h || !bytes) return CL_ERR_ARG;
    *bytes = h->c.device_bytes;
    return CL_OK;
}

int cl_upload_mask(cl_ctx* h, const uint8_t* mask) {
    if (!h || !mask) { set_error("null argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    CL_CUDA(cudaMemcpyAsync(c->d_mask, mask, c->geo.N, cudaMemcpyHostToDevice, c->stream));
    int r = phase_seed(c);
    if (r) return r;
    r = classes_from_mask(c);
    if (r) return r;
    c->mask_ready = true;
    return CL_OK;
}

int cl_download_mask(cl_ctx* h, uint8_t* mask) {
    if (!h || !mask) { set_error("null argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    CL_CUDA(cudaMemcpyAsync(mask, c->d_mask, c->geo.N, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

int cl_flow_init(cl_ctx* h) {
    if (!h) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->mask_ready) { set_error("upload the mask first"); return CL_ERR_STATE; }
    int r = flow_init(c);
    if (r) return r;
    c->flow_ready = true;
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

// Runs of flow steps are replayed from a CUDA graph: a chunk of
// kFlowGraphSteps steps (an even number, so the AA parity comes back) is
// captured once per FlowGraphKey and launched as one graph, so a small
// lattice steps at the kernels' pace instead of the host's launch rate.
// Timed runs (cl_timing) and contexts on the legacy default stream launch
// step by step.
constexpr int kFlowGraphSteps = 32;

static FlowGraphKey flow_key(const Ctx* c, int use_tracer) {
    FlowGraphKey k{};
    k.f = c->d_f; k.list = c->d_flive; k.sidx = c->d_fsidx; k.cls = c->d_ns_cls; k.tracer = c->d_tracer;
    k.part = c->d_energy_part; k.count = c->n_flive; k.n_bgk = c->n_bgk;
    k.tau_ns = c->cfg.tau_ns; k.perm_ratio = c->cfg.perm_ratio; k.rho_in = c->cfg.rho_in; k.rho_out = c->cfg.rho_out;
    k.energy_blocks = c->energy_blocks; k.nodyn_coupled = c->flow_nodyn_coupled ? 1 : 0; k.use_tracer = use_tracer;
    k.parity = c->flow_parity; k.stream = c->stream;
    return k;
}

static bool same_key(const FlowGraphKey& a, const FlowGraphKey& b) {
    return a.f == b.f && a.list == b.list && a.sidx == b.sidx && a.cls == b.cls && a.tracer == b.tracer &&
           a.part == b.part && a.count == b.count && a.n_bgk == b.n_bgk && a.tau_ns == b.tau_ns &&
           a.perm_ratio == b.perm_ratio && a.rho_in == b.rho_in && a.rho_out == b.rho_out &&
           a.energy_blocks == b.energy_blocks && a.nodyn_coupled == b.nodyn_coupled &&
           a.use_tracer == b.use_tracer && a.parity == b.parity && a.stream == b.stream;
}

static int flow_graph_ready(Ctx* c, int use_tracer) {
    const FlowGraphKey key = flow_key(c, use_tracer);
    if (c->flow_graph && same_key(key, c->flow_graph_key)) return CL_OK;
    if (c->flow_graph) { cudaGraphExecDestroy(c->flow_graph); c->flow_graph = nullptr; }
    CL_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    const int64_t launches0 = c->launches;
    const int parity0 = c->flow_parity;
    int r = CL_OK;
    for (int s = 0; s < kFlowGraphSteps && !r; ++s) r = flow_step(c, use_tracer);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    c->launches = launches0;                 // nothing ran yet
    c->flow_parity = parity0;
    if (r) { if (g) cudaGraphDestroy(g); return r; }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t ei = cudaGraphInstantiate(&c->flow_graph, g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) { c->flow_graph = nullptr; return cuda_fail(ei, "cudaGraphInstantiate"); }
    c->flow_graph_key = key;
    return CL_OK;
}

static int run_flow(Ctx* c, int32_t n, int use_tracer) {
    int32_t i = 0;
    // a step that brings the storage or the list up to date runs plainly
    while (i < n && (c->fstore_dirty || c->flive_dirty)) {
        int r = flow_step(c, use_tracer);
        if (r) return r;
        ++i;
    }
    if (!c->timing && c->stream != nullptr && n - i >= kFlowGraphSteps) {
        int r = flow_graph_ready(c, use_tracer);
        if (r) return r;
        for (; n - i >= kFlowGraphSteps; i += kFlowGraphSteps) {
            CL_CUDA(cudaGraphLaunch(c->flow_graph, c->stream));
            c->launches += 2 * kFlowGraphSteps;
        }
    }
    for (; i < n; ++i) {
        int r = flow_step(c, use_tracer);
        if (r) return r;
    }
    return CL_OK;
}

// after a synchronising call: a flow site that streamed without the storage it
// needed (counted by the step) is an error
static int flow_storage_check(Ctx* c) {
    unsigned long long cnt = 0;
    CL_CUDA(cudaMemcpyAsync(&cnt, c->d_counters + 2, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaMemsetAsync(c->d_counters + 2, 0, sizeof cnt, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    if (cnt) { set_error("flow step: a streaming site's slots had no storage"); return CL_ERR_STATE; }
    return CL_OK;
}

int cl_flow_steps(cl_ctx* h, int32_t n) {
    if (!h || n < 0) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->flow_ready) { set_error("call cl_flow_init first"); return CL_ERR_STATE; }
    int r = flow_arm_tracer(c, 0.0);
    if (r) return r;
    if ((r = run_flow(c, n, 0))) return r;
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return flow_storage_check(c);
}

int cl_flow_solve(cl_ctx* h, int32_t max_it, double eps, int32_t* iters) {
    if (!h || max_it < 0) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->flow_ready) { set_error("call cl_flow_init first"); return CL_ERR_STATE; }
    int r = flow_arm_tracer(c, eps);
    if (r) return r;
    const int chunk = 200;
    int done = 0;
    FlowTracer tr;
    while (done < max_it) {
        const int n = (max_it - done) < chunk ? (max_it - done) : chunk;
        // launch n steps; once converged the remaining launches exit at once
        if ((r = run_flow(c, n, 1))) return r;
        CL_CUDA(cudaMemcpyAsync(&tr, c->d_tracer, sizeof tr, cudaMemcpyDeviceToHost, c->stream));
        CL_CUDA(cudaStreamSynchronize(c->stream));
        done += n;
        if (tr.converged) break;
    }
    CL_CUDA(cudaMemcpyAsync(&tr, c->d_tracer, sizeof tr, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    if ((r = flow_storage_check(c))) return r;
    // parity follows the steps actually executed
    c->flow_parity = tr.steps_done & 1;
    // the reference's loop counter at exit: the index of the converging step, or max_it
    if (iters) *iters = tr.converged ? (tr.converged_at - 1) : max_it;
    if (tr.diverged) { set_error("flow diverged (NaN energy)"); return CL_ERR_DIVERGED; }
    return tr.converged ? CL_OK : CL_WARN_NOT_CONVERGED;
}

int cl_flow_energy(cl_ctx* h, double* energy) {
    if (!h || !energy) return CL_ERR_ARG;
    Ctx* c = &h->c;
    FlowTracer tr;
    CL_CUDA(cudaMemcpyAsync(&tr, c->d_tracer, sizeof tr, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    *energy = tr.last_energy;
    return CL_OK;
}

int cl_couple_velocity(cl_ctx* h) {
    if (!h) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->flow_ready) { set_error("no flow field"); return CL_ERR_STATE; }
    int r = flow_macro(c, nullptr, c->d_u, 1);
    if (r) return r;
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

int cl_flow_velocity_stats(cl_ctx* h, double* pore_mean_u, double* max_ux, double* outlet_mean_ux) {
    if (!h) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->flow_ready) { set_error("no flow field"); return CL_ERR_STATE; }
    double v[3];
    int r = flow_stats(c, v);
    if (r) return r;
    const double box = (double)(c->geo.N - 2 * c->geo.plane), plane = (double)c->geo.plane;
    if (pore_mean_u) *pore_mean_u = v[0] / box;
    if (max_ux) *max_ux = v[1];
    if (outlet_mean_ux) *outlet_mean_ux = v[2] / plane;
    return CL_OK;
}

int cl_flow_velocity_norm_masked(cl_ctx* h, int32_t code, double* sum_norm, int64_t* count) {
    if (!h || code < 0 || code > 255) { set_error("cl_flow_velocity_norm_masked: bad argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    if (!c->flow_ready) { set_error("no flow field"); return CL_ERR_STATE; }
    double v[2];
    int r = flow_norm_masked(c, code, v);
    if (r) return r;
    if (sum_norm) *sum_norm = v[0];
    if (count) *count = (int64_t)(v[1] + 0.5);
    return CL_OK;
}

int cl_set_flow_pressure(cl_ctx* h, double rho_in, double rho_out) {
    if (!h || !(rho_in > 0.0) || !(rho_out > 0.0)) { set_error("cl_set_flow_pressure: densities must be positive"); return CL_ERR_ARG; }
    h->c.cfg.rho_in = rho_in;
    h->c.cfg.rho_out = rho_out;
    return CL_OK;
}

int cl_set_transport(cl_ctx* h, const double* omega_pore, const double* omega_bio, double dt) {
    if (!h || !omega_pore || !omega_bio || !(dt > 0.0)) { set_error("cl_set_transport: bad argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    for (int s = 0; s < c->cfg.n_solutes; ++s) {
        if (c->ap.mob_slot[s] < 0) continue;     // an immobile solute has no lattice to relax (D = 0 gives 2)
        if (!(omega_pore[s] > 0.0 && omega_pore[s] < 2.0) || !(omega_bio[s] > 0.0 && omega_bio[s] < 2.0)) {
            set_error("cl_set_transport: relaxation frequencies must lie in (0, 2)"); return CL_ERR_ARG;
        }
    }
    for (int s = 0; s < c->cfg.n_solutes; ++s) {
        c->cfg.omega_pore[s] = omega_pore[s];
        c->cfg.omega_bio[s] = omega_bio[s];
        const int m = c->ap.mob_slot[s];
        if (m >= 0) { c->ap.omega_pore[m] = (float)omega_pore[s]; c->ap.omega_bio[m] = (float)omega_bio[s]; }
    }
    c->cfg.dt = dt;
    c->ap.dt = dt;
    return CL_OK;
}

int cl_update_dynamics(cl_ctx* h) {
    if (!h) return CL_ERR_ARG;
    return update_dynamics(&h->c);
}

int cl_ade_init(cl_ctx* h) {
    if (!h) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->mask_ready) { set_error("upload the mask first"); return CL_ERR_STATE; }
    int r = ade_init(c);
    if (r) return r;
    if ((r = phase_fill(c))) return r;
    if ((r = ca_init(c))) return r;
    c->ade_ready = true;
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

int cl_set_surrogate(cl_ctx* h, int32_t slot, const cl_surrogate_net* net) {
    if (!h || !net || slot < 0 || slot >= CL_MAX_SRG_ORG) { set_error("cl_set_surrogate: bad argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    SrgNetDev d{};
    d.L = net->n_layers;
    if (d.L < 1 || d.L > CL_SRG_MAX_LAYERS) { set_error("surrogate: 1..5 layers"); return CL_ERR_ARG; }
    int off = 0;
    for (int l = 0; l <= d.L; ++l) {
        d.w[l] = net->widths[l];
        if (d.w[l] < 1 || d.w[l] > CL_SRG_MAX_WIDTH) { set_error("surrogate: widths 1..32"); return CL_ERR_ARG; }
    }
    for (int l = 0; l < d.L; ++l) { d.poff[l] = off; off += d.w[l + 1] * d.w[l] + d.w[l + 1]; }
    if (off > 4096) { set_error("surrogate: too many parameters"); return CL_ERR_ARG; }
    for (int i = 0; i < CL_SRG_MAX_WIDTH; ++i) {
        d.xo[i] = (float)net->x_offset[i]; d.xg[i] = (float)net->x_gain[i];
        d.xlo[i] = (float)std::max(net->x_lo[i], -3.0e38); d.xhi[i] = (float)std::min(net->x_hi[i], 3.0e38);
        d.yo[i] = (float)net->y_offset[i]; d.yg[i] = (float)net->y_gain[i];
    }
    d.xymin = (float)net->x_ymin; d.yymin = (float)net->y_ymin;
    std::vector<float> hp(off);
    for (int i = 0; i < off; ++i) hp[i] = (float)net->params[i];
    if (c->d_srg_params[slot]) { cudaFree(c->d_srg_params[slot]); c->d_srg_params[slot] = nullptr; }
    int r = dalloc(c, &c->d_srg_params[slot], (size_t)off);
    if (r) return r;
    CL_CUDA(cudaMemcpyAsync(c->d_srg_params[slot], hp.data(), sizeof(float) * off, cudaMemcpyHostToDevice, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    d.params = c->d_srg_params[slot];
    c->ap.net[slot] = d;
    c->h_srg_params[slot] = std::move(hp);
    return CL_OK;
}

// learning on (interval > 0) or off: the network and its ring of pairs
static int learn_enable(Ctx* c, int64_t interval) {
    if (interval < 0 || interval > (1 << 30)) { set_error("cl_set_option: learning interval >= 0"); return CL_ERR_ARG; }
    if (interval == 0) { c->learn_interval = 0; return CL_OK; }
    const cl_eq_system& e = c->cfg.eq;
    if (!c->cfg.use_equilibrium || e.solver != CL_EQ_SOLVER_NEWTON || e.n_comp > 5 || c->chem == 0 || !c->chem_on) {
        set_error("the learned start needs Newton speciation (1..5 components) in a compiled chemistry's step");
        return CL_ERR_STATE;
    }
    if (!c->learn) {
        int st = CL_OK;
        c->learn = cl_eq_create(&e, c->stream, &st);
        if (!c->learn) return st;
        c->pair_cap = 1 << 20;
        int r = CL_OK;
        if ((r = dalloc(c, &c->d_pair_T, (size_t)c->pair_cap * e.n_comp)) ||
            (r = dalloc(c, &c->d_pair_X, (size_t)c->pair_cap * e.n_comp)) || (r = dalloc(c, &c->d_pair_count, 1)))
            return r;
        CL_CUDA(cudaMemsetAsync(c->d_pair_count, 0, sizeof(unsigned long long), c->stream));
    }
    c->learn_interval = (int)interval;
    c->learn_steps = 0;
    return CL_OK;
}

// after a step: every learn_interval steps, train on the ring and empty it
static int learn_after_step(Ctx* c) {
    if (!c->learn || c->learn_interval <= 0) return CL_OK;
    if (++c->learn_steps < c->learn_interval) return CL_OK;
    c->learn_steps = 0;
    unsigned long long cnt = 0;
    CL_CUDA(cudaMemcpyAsync(&cnt, c->d_pair_count, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    const int64_t n = std::min<int64_t>((int64_t)cnt, c->pair_cap);
    if (n < 4096) return CL_OK;                 // fewer than one training batch: keep collecting
    float loss = 0.f;
    int r = cl_eq_train(c->learn, c->d_pair_T, c->d_pair_X, n, c->learn_epochs, 4096, 3e-3f,
                        (uint64_t)c->step_index, &loss);
    if (r < 0) return r;
    c->learn_loss = loss;
    c->learn_ready = true;
    ++c->learn_trainings;
    CL_CUDA(cudaMemsetAsync(c->d_pair_count, 0, sizeof(unsigned long long), c->stream));
    return CL_OK;
}

int cl_set_option(cl_ctx* h, int32_t key, int64_t value) {
    if (!h) return CL_ERR_ARG;
    Ctx* c = &h->c;
    switch (key) {
        case CL_OPT_COMPILED_CHEM:
            if (value == 0 && c->cfg.rate_law != CL_RATELAW_TABLE) {
                set_error("cl_set_option: a compiled rate law has no run-time table form");
                return CL_ERR_ARG;
            }
            c->chem_on = value != 0;
            return CL_OK;
        case CL_OPT_FAST_VARIANT:
            if (value < 0 || value > 3) { set_error("cl_set_option: variant 0..3"); return CL_ERR_ARG; }
            c->fast_variant = (int)value; return CL_OK;
        case CL_OPT_EQ_LEARN: return learn_enable(c, value);
        case CL_OPT_EQ_FORGET: {
            const int nc = c->cfg.eq.n_comp;
            if (c->d_eq_x) CL_CUDA(cudaMemsetAsync(c->d_eq_x, 0xff, sizeof(float) * nc * c->geo.N, c->stream));
            if (c->d_eq_xp) CL_CUDA(cudaMemsetAsync(c->d_eq_xp, 0xff, sizeof(float) * nc * c->geo.N, c->stream));
            CL_CUDA(cudaStreamSynchronize(c->stream));
            return CL_OK;
        }
        default: set_error("cl_set_option: unknown key"); return CL_ERR_ARG;
    }
}

int cl_get_option(cl_ctx* h, int32_t key, int64_t* value) {
    if (!h || !value) return CL_ERR_ARG;
    Ctx* c = &h->c;
    switch (key) {
        case CL_OPT_COMPILED_CHEM: *value = c->chem_on ? c->chem : 0; return CL_OK;
        case CL_OPT_FAST_VARIANT: *value = c->fast_variant; return CL_OK;
        case CL_OPT_EQ_LEARN: *value = c->learn_interval; return CL_OK;
        case CL_OPT_EQ_LEARN_TRAININGS: *value = c->learn_trainings; return CL_OK;
        default: set_error("cl_get_option: unknown key"); return CL_ERR_ARG;
    }
}

int cl_op_collide(cl_ctx* h) { return h ? ops_collide(&h->c) : CL_ERR_ARG; }
int cl_op_stream(cl_ctx* h) { return h ? ops_stream(&h->c) : CL_ERR_ARG; }
int cl_op_reactions(cl_ctx* h, int32_t ops) {
    if (!h || ops < 0 || ops > CL_OP_ALL) { set_error("cl_op_reactions: ops is a mask of CL_OP_*"); return CL_ERR_ARG; }
    return ops ? ops_react(&h->c, ops) : CL_OK;
}
int cl_op_kinetics(cl_ctx* h) { return cl_op_reactions(h, CL_OP_KINETICS); }
int cl_op_surrogate(cl_ctx* h) { return cl_op_reactions(h, CL_OP_SURROGATE); }
int cl_op_abiotic(cl_ctx* h) { return cl_op_reactions(h, CL_OP_ABIOTIC); }
int cl_op_equilibrium(cl_ctx* h) { return cl_op_reactions(h, CL_OP_EQUILIBRIUM); }

int cl_step(cl_ctx* h, int32_t n) {
    if (!h || n < 0) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
    if (c->op_collided) { set_error("cl_step between cl_op_collide and cl_op_stream"); return CL_ERR_STATE; }
    for (int o = 0; o < c->ap.n_srg; ++o)
        if (!c->ap.net[c->ap.srg[o].net].params) { set_error("surrogate network slot not set"); return CL_ERR_STATE; }
    if (c->ap.n_mob == 0) { set_error("no mobile solute"); return CL_ERR_STATE; }
    for (int32_t i = 0; i < n; ++i) {
        int r = ade_step(c);
        if (r) return r;
        ++c->step_index;
        if ((r = learn_after_step(c))) return r;
    }
    unsigned long long cnts[2] = {0, 0};
    CL_CUDA(cudaMemcpyAsync(cnts, c->d_counters, sizeof cnts, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaMemsetAsync(c->d_counters, 0, sizeof cnts, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    if (cnts[1]) { set_error("transport step: a live site's slots had no storage"); return CL_ERR_STATE; }
    return cnts[0] ? CL_WARN_NOT_CONVERGED : CL_OK;
}

}  // extern "C"

namespace cl {

__global__ void f2d_kernel(const float* a, double* b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = a[i];
}
__global__ void d2f_kernel(const double* a, float* b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = (float)a[i];
}
__global__ void i2d_kernel(const int32_t* a, double* b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = a[i];
}
__global__ void u2d_kernel(const uint8_t* a, double* b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = a[i];
}
// dynamics classes (the low two bits of a class byte) <-> doubles; a value
// that is not a class 0..3 sets *bad and leaves the byte as it was
__global__ void cls2d_kernel(const uint8_t* a, double* b, int64_t n) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) b[i] = a[i] & 3;
}
__global__ void d2cls_kernel(const double* a, uint8_t* b, int64_t n, int* bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = a[i];
        if (v >= 0.0 && v <= 3.0 && v == (double)(int)v) b[i] = (uint8_t)((b[i] & ~3) | (int)v);
        else *bad = 1;
    }
}
// phase ids from doubles; any value that is not an id 0..n_phases sets *bad
__global__ void d2phase_kernel(const double* a, uint8_t* b, int64_t n, int n_phases, int* bad) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double v = a[i];
        if (v >= 0.0 && v <= (double)n_phases && v == (double)(int)v) b[i] = (uint8_t)(int)v;
        else { b[i] = 0; *bad = 1; }
    }
}
// set solute populations to t_i * c at the slots that hold each site's
// pre-collision populations for the current parity
// every site is stored when this runs (cl_set_field stores them all first)
template <int PARITY>
__global__ void ade_set_kernel(Geo g, float* pm, const int32_t* sidx, const double* c) {
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t n = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; n < g.N; n += stride) {
        int x, y, z;
        decode(g, n, x, y, z);
        const float v = (float)c[n];
        const int32_t sn = sidx[n];
        if (sn < 0) continue;
#pragma unroll
        for (int i = 0; i < 7; ++i) {
            if (PARITY == 0) pm[i * g.N + sn] = t7(i) * v;
            else {
                const int64_t m = nbr(g, n, x, y, z, -c7x(i), -c7y(i), -c7z(i));
                const int32_t sm = m < 0 ? -1 : sidx[m];
                if (m < 0) pm[i * g.N + sn] = t7(i) * v;
                else if (sm >= 0) pm[opp7(i) * g.N + sm] = t7(i) * v;
            }
        }
    }
}

}  // namespace cl

extern "C" {

int cl_get_field(cl_ctx* h, int32_t field, int32_t index, double* out) {
    if (!h || !out) { set_error("null argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    const int64_t N = c->geo.N;
    double* d = c->d_scratch;
    const int blocks = grid_for(N, 256, 148 * 16);
    int r = CL_OK;
    switch (field) {
        case CL_FIELD_CONC:
            if (index < 0 || index >= c->ap.S || !c->ade_ready) { set_error("bad solute / not initialised"); return CL_ERR_ARG; }
            r = ade_density(c, index, d); break;
        case CL_FIELD_BIOMASS:
            if (index < 0 || index >= c->ap.M) { set_error("bad microbe"); return CL_ERR_ARG; }
            CL_CUDA(cudaMemcpyAsync(d, c->d_bio + (int64_t)index * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
            break;
        case CL_FIELD_VELOCITY:
            if (index < 0 || index > 2) return CL_ERR_ARG;
            f2d_kernel<<<blocks, 256, 0, c->stream>>>(c->d_u + index * N, d, N);
            break;
        case CL_FIELD_FLOW_RHO:
            if (!c->flow_ready) return CL_ERR_STATE;
            r = flow_macro(c, d, nullptr, 1); break;
        case CL_FIELD_FLOW_U: {
            if (index < 0 || index > 2 || !c->flow_ready) return CL_ERR_ARG;
            // computes all three into the velocity buffer's shape in scratch (floats)
            float* fu = reinterpret_cast<float*>(d + N / 2 + 1);
            if (3 * N * sizeof(float) > (N / 2) * sizeof(double)) {
                // not enough room after the output: go through the coupled-velocity buffer copy
                float* tmp = nullptr;
                CL_CUDA(cudaMalloc(&tmp, sizeof(float) * 3 * N));
                r = flow_macro(c, nullptr, tmp, 1);
                if (!r) f2d_kernel<<<blocks, 256, 0, c->stream>>>(tmp + index * N, d, N);
                cudaStreamSynchronize(c->stream);
                cudaFree(tmp);
            } else {
                r = flow_macro(c, nullptr, fu, 1);
                if (!r) f2d_kernel<<<blocks, 256, 0, c->stream>>>(fu + index * N, d, N);
            }
            break;
        }
        case CL_FIELD_EQ_ITERS:
            if (!c->d_eq_iters) return CL_ERR_STATE;
            i2d_kernel<<<blocks, 256, 0, c->stream>>>(c->d_eq_iters, d, N);
            break;
        case CL_FIELD_EQ_START:
            if (!c->ade_ready) return CL_ERR_STATE;
            r = eq_start_io(c, index, d, 1);
            break;
        case CL_FIELD_DYNAMICS:
            if (!c->mask_ready || index < 0 || index > 1) { set_error("dynamics: index 0 (flow) or 1 (transport), after the mask"); return CL_ERR_ARG; }
            cls2d_kernel<<<blocks, 256, 0, c->stream>>>(index == 0 ? c->d_ns_cls : c->d_ade_cls, d, N);
            break;
        case CL_FIELD_PHASE:
            if (!c->d_phase) { set_error("dissolution is not enabled in this context"); return CL_ERR_STATE; }
            u2d_kernel<<<blocks, 256, 0, c->stream>>>(c->d_phase, d, N);
            break;
        case CL_FIELD_CA_AGE:
        case CL_FIELD_CA_TOTAL:
            if (!c->ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
            r = ca_field(c, field, d); break;
        default: set_error("unknown field"); return CL_ERR_ARG;
    }
    if (r) return r;
    CL_LAUNCH_CHECK("cl_get_field");
    CL_CUDA(cudaMemcpyAsync(out, d, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

int cl_set_field(cl_ctx* h, int32_t field, int32_t index, const double* in) {
    if (!h || !in) { set_error("null argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    const int64_t N = c->geo.N;
    double* d = c->d_scratch;
    const int blocks = grid_for(N, 256, 148 * 16);
    CL_CUDA(cudaMemcpyAsync(d, in, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
    switch (field) {
        case CL_FIELD_CONC: {
            if (index < 0 || index >= c->ap.S || !c->ade_ready) { set_error("bad solute / not initialised"); return CL_ERR_ARG; }
            const int slot = c->ap.mob_slot[index];
            if (slot < 0) {
                CL_CUDA(cudaMemcpyAsync(c->d_imm + (int64_t)index * N, d, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
            } else {
                // densities may be set anywhere, so every site gets storage
                // (this uses the scratch, so the input is copied again after)
                int r2 = store_update(c, 1);
                if (r2) return r2;
                CL_CUDA(cudaMemcpyAsync(d, in, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
                float* pm = c->d_g + (int64_t)slot * 7 * N;
                if (c->ade_parity == 0) ade_set_kernel<0><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, d);
                else ade_set_kernel<1><<<blocks, 256, 0, c->stream>>>(c->geo, pm, c->d_sidx, d);
            }
            break;
        }
        case CL_FIELD_BIOMASS:
            if (index < 0 || index >= c->ap.M) { set_error("bad microbe"); return CL_ERR_ARG; }
            CL_CUDA(cudaMemcpyAsync(c->d_bio + (int64_t)index * N, d, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream));
            break;
        case CL_FIELD_VELOCITY:
            if (index < 0 || index > 2) return CL_ERR_ARG;
            d2f_kernel<<<blocks, 256, 0, c->stream>>>(d, c->d_u + index * N, N);
            break;
        case CL_FIELD_DYNAMICS: {
            if (!c->mask_ready || index < 0 || index > 1) { set_error("dynamics: index 0 (flow) or 1 (transport), after the mask"); return CL_ERR_ARG; }
            int* d_bad = reinterpret_cast<int*>(c->d_scratch + N);
            CL_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), c->stream));
            d2cls_kernel<<<blocks, 256, 0, c->stream>>>(d, index == 0 ? c->d_ns_cls : c->d_ade_cls, N, d_bad);
            CL_LAUNCH_CHECK("d2cls_kernel");
            int bad = 0;
            CL_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, c->stream));
            CL_CUDA(cudaStreamSynchronize(c->stream));
            // the flags, counts, site lists and storage follow the classes
            const int r2 = refresh_flags(c);
            if (r2) return r2;
            if (bad) { set_error("dynamics classes are 0 NoDynamics, 1 bounce-back, 2 pore, 3 biofilm"); return CL_ERR_ARG; }
            break;
        }
        case CL_FIELD_EQ_START: {
            if (!c->ade_ready) return CL_ERR_STATE;
            // storage first (its update uses the scratch that holds the input),
            // then the input again
            if (c->store_dirty) {
                const int r2 = store_update(c, 0);
                if (r2) return r2;
                CL_CUDA(cudaMemcpyAsync(d, in, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
            }
            const int r2 = eq_start_io(c, index, d, 0);
            if (r2) return r2;
            break;
        }
        case CL_FIELD_PHASE: {
            if (!c->d_phase) { set_error("dissolution is not enabled in this context"); return CL_ERR_STATE; }
            int* d_bad = reinterpret_cast<int*>(c->d_scratch + N);
            CL_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), c->stream));
            d2phase_kernel<<<blocks, 256, 0, c->stream>>>(d, c->d_phase, N, c->cfg.n_phases, d_bad);
            CL_LAUNCH_CHECK("d2phase_kernel");
            int bad = 0;
            CL_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, c->stream));
            CL_CUDA(cudaStreamSynchronize(c->stream));
            int r = refresh_flags(c);
            if (r) return r;
            if (bad) { set_error("phase ids must be integers 0..n_phases (others were set to 0)"); return CL_ERR_ARG; }
            break;
        }
        default: set_error("field is read-only or unknown"); return CL_ERR_ARG;
    }
    CL_LAUNCH_CHECK("cl_set_field");
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return CL_OK;
}

int cl_get_flow_populations(cl_ctx* h, float* out) {
    if (!h || !out) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->flow_ready) { set_error("no flow field"); return CL_ERR_STATE; }
    const int64_t N = c->geo.N;
    float* tmp = nullptr;
    CL_CUDA(cudaMalloc(&tmp, sizeof(float) * 19 * N));
    int r = flow_population_io(c, tmp, 1);
    if (!r) {
        cudaError_t e = cudaMemcpyAsync(out, tmp, sizeof(float) * 19 * N, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "cl_get_flow_populations");
    }
    cudaFree(tmp);
    return r;
}

int cl_set_flow_populations(cl_ctx* h, const float* in) {
    if (!h || !in) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->mask_ready) { set_error("upload the mask first"); return CL_ERR_STATE; }
    const int64_t N = c->geo.N;
    float* tmp = nullptr;
    CL_CUDA(cudaMalloc(&tmp, sizeof(float) * 19 * N));
    cudaError_t e = cudaMemcpyAsync(tmp, in, sizeof(float) * 19 * N, cudaMemcpyHostToDevice, c->stream);
    int r = e == cudaSuccess ? flow_population_io(c, tmp, 0) : cuda_fail(e, "cl_set_flow_populations");
    if (!r) { e = cudaStreamSynchronize(c->stream); if (e != cudaSuccess) r = cuda_fail(e, "sync"); }
    cudaFree(tmp);
    if (!r) c->flow_ready = true;
    return r;
}

int cl_set_solute_populations(cl_ctx* h, int32_t s, const float* in) {
    if (!h || !in) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (!c->ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
    if (s < 0 || s >= c->ap.S || c->ap.mob_slot[s] < 0) { set_error("not a mobile solute"); return CL_ERR_ARG; }
    const int64_t N = c->geo.N;
    float* tmp = nullptr;
    CL_CUDA(cudaMalloc(&tmp, sizeof(float) * 7 * N));
    cudaError_t e = cudaMemcpyAsync(tmp, in, sizeof(float) * 7 * N, cudaMemcpyHostToDevice, c->stream);
    int r = e == cudaSuccess ? ade_population_set(c, c->ap.mob_slot[s], tmp) : cuda_fail(e, "cl_set_solute_populations");
    cudaFree(tmp);
    return r;
}

int cl_get_solute_populations(cl_ctx* h, int32_t s, float* out) {
    if (!h || !out) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (s < 0 || s >= c->ap.S || c->ap.mob_slot[s] < 0) { set_error("not a mobile solute"); return CL_ERR_ARG; }
    const int64_t N = c->geo.N;
    float* tmp = nullptr;
    CL_CUDA(cudaMalloc(&tmp, sizeof(float) * 7 * N));
    int r = ade_population_io(c, c->ap.mob_slot[s], tmp);
    if (!r) {
        cudaError_t e = cudaMemcpyAsync(out, tmp, sizeof(float) * 7 * N, cudaMemcpyDeviceToHost, c->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = cuda_fail(e, "cl_get_solute_populations");
    }
    cudaFree(tmp);
    return r;
}

int cl_reduce(cl_ctx* h, int32_t field, int32_t index, int32_t op, double arg, double* out) {
    if (!h || !out) { set_error("null argument"); return CL_ERR_ARG; }
    Ctx* c = &h->c;
    if (op == CL_RED_COUNT_EQ) return reduce_field(c, nullptr, op, arg, c->d_mask, out);
    if (op < 0 || op > 2) return CL_ERR_ARG;
    // materialise the field into the first N doubles of scratch, reduce from a copy region
    double* tmp = nullptr;
    const int64_t N = c->geo.N;
    CL_CUDA(cudaMalloc(&tmp, sizeof(double) * N));
    int r = CL_OK;
    switch (field) {
        case CL_FIELD_CONC: r = (index >= 0 && index < c->ap.S) ? ade_density(c, index, tmp) : CL_ERR_ARG; break;
        case CL_FIELD_BIOMASS:
            if (index < 0 || index >= c->ap.M) r = CL_ERR_ARG;
            else { cudaError_t e = cudaMemcpyAsync(tmp, c->d_bio + (int64_t)index * N, sizeof(double) * N, cudaMemcpyDeviceToDevice, c->stream);
                   if (e != cudaSuccess) r = cuda_fail(e, "copy"); }
            break;
        case CL_FIELD_FLOW_RHO: r = flow_macro(c, tmp, nullptr, 1); break;
        default: r = CL_ERR_ARG; set_error("field not reducible");
    }
    if (!r) r = reduce_field(c, tmp, op, arg, nullptr, out);
    cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    return r;
}

int cl_timing_enable(cl_ctx* h, int32_t on) {
    if (!h) return CL_ERR_ARG;
    Ctx* c = &h->c;
    if (on && !c->ev[0][0][0]) {
        for (int k = 0; k < Ctx::kTimedKernels; ++k)
            for (int i = 0; i < Ctx::kEventPool; ++i)
                for (int j = 0; j < 2; ++j) CL_CUDA(cudaEventCreate(&c->ev[k][i][j]));
    }
    c->timing = on != 0;
    return CL_OK;
}

int cl_timing_read(cl_ctx* h, int32_t kernel, double* total_ms, int64_t* launches) {
    if (!h || kernel < 0 || kernel >= Ctx::kTimedKernels) return CL_ERR_ARG;
    Ctx* c = &h->c;
    CL_CUDA(cudaStreamSynchronize(c->stream));
    int r = timing_end(c, -1 - kernel);   // fold the pending pairs
    if (r) return r;
    if (total_ms) *total_ms = c->ev_ms[kernel];
    if (launches) *launches = c->ev_launches[kernel];
    c->ev_ms[kernel] = 0.0;
    c->ev_launches[kernel] = 0;
    return CL_OK;
}

int cl_launch_count(const cl_ctx* h, int64_t* launches) {
    if (!h || !launches) return CL_ERR_ARG;
    *launches = h->c.launches;
    return CL_OK;
}

int cl_precip_convert(cl_ctx* h, int64_t* changed) {
    if (!h || !changed) return CL_ERR_ARG;
    return precip_convert(&h->c, changed);
}

int cl_dissol_convert(cl_ctx* h, int64_t* changed) {
    if (!h || !changed) return CL_ERR_ARG;
    return dissol_convert(&h->c, changed);
}

int cl_ca_update_mask(cl_ctx* h, int64_t* mask_changes) {
    if (!h) return CL_ERR_ARG;
    if (!h->c.ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
    return ca_update_mask(&h->c, mask_changes);
}

int cl_fd_diffuse(cl_ctx* h, double nu, uint32_t microbes) {
    if (!h || !(nu >= 0.0) || !std::isfinite(nu)) { set_error("cl_fd_diffuse: bad argument"); return CL_ERR_ARG; }
    if (!h->c.ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
    if (h->c.cfg.n_microbes < 32 && (microbes >> h->c.cfg.n_microbes) != 0u) {
        set_error("cl_fd_diffuse: a selected microbe does not exist");
        return CL_ERR_ARG;
    }
    return fd_diffuse(&h->c, nu, microbes);
}

int cl_ca_redistribute(cl_ctx* h, int32_t* sweeps, int64_t* mask_changes, double* bmax_after) {
    if (!h) return CL_ERR_ARG;
    if (!h->c.ade_ready) { set_error("call cl_ade_init first"); return CL_ERR_STATE; }
    return ca_redistribute(&h->c, sweeps, mask_changes, bmax_after);
}

}  // extern "C"
