// complab_main.cpp -- host driver: CompLaB.xml in, the reference's time loop
// (src/complab.cpp:560-1860) over the C ABI, fields out.
//
//   complab_b200 [CompLaB.xml] [--steps N] [--eq-solver newton|pcf] [--rates rates.xml]
//                [--restart DIR] [--dump-config FILE] [--print-config] [--quiet]
//
// Output: at every <save_VTK_interval> and at the end, the fields as raw FP64
// arrays and as the reference's VTI files; at every <save_CHK_interval> a
// checkpoint folder chk_<steps>/ (formats: complab_io.h), which --restart
// resumes from (the configuration still comes from CompLaB.xml).
//
// --rates supplies the rate-law blocks (<rate_table>, dissolution <rate_k> ...)
// that the main file lacks; --dump-config writes the cl_config the transport
// loop starts from (after the Peclet calibration) as raw bytes to FILE and the
// geometry as read to FILE.mask, so that a checker can replay the run.
//
// --eq-solver pcf runs the reference's live speciation solver (PCF + Anderson)
// in the transport step; the default is Newton (or the XML's <solver>).
//
// Order, as main() of the reference runs it:
//   read CompLaB.xml and the geometry (readGeometry, complab_functions.hh:127-156);
//   flow to steady state with the ValueTracer (complab.cpp:614-620); if a Peclet
//   number is set, the permeability from the outlet Darcy velocity, a corrected
//   deltaP and a second solve (:641-669);
//   solute relaxation and dt from the flow (:708-727), velocity coupling (:1096-1101);
//   then per transport step: collide .. kinetics .. abiotic (+ dissolution) ..
//   equilibrium .. stream (cl_step); the cellular-automaton biomass
//   redistribution (:1453-1715) with its dynamics switch and flow re-solve on a
//   mask change (:1734-1780); on their intervals the precipitation and
//   dissolution node conversions with the dynamics switch, flow re-solve and
//   re-coupling (:1783-1845).
// Fields are written as raw little-endian FP64 arrays in site order
// n = (x*ny + y)*nz + z, one file per solute (and microbe) per output step,
// with a JSON index; the run summary goes to stdout as one JSON line.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>
#include <sstream>
#include <map>

#include "../../include/complab_gpu.h"
#include "complab_io.h"
#include "complab_xml.h"

using clhost::HostRun;

namespace {

constexpr double kThrd = 1e-12;

struct Ctx {
    cl_ctx* h = nullptr;
    ~Ctx() { if (h) cl_destroy(h); }
};

bool check(int st, const char* what) {
    if (st < 0) {
        std::fprintf(stderr, "complab_b200: %s failed (%d): %s\n", what, st, cl_last_error());
        return false;
    }
    return true;
}

// readGeometry: nx-2 slices of ny*nz integers (y-major, z fastest); the
// boundary planes repeat the first and last slice
bool read_geometry(const std::string& file, int nx, int ny, int nz, std::vector<uint8_t>& mask, std::string& err) {
    std::ifstream f(file);
    if (!f) { err = "could not open geometry file " + file; return false; }
    const size_t plane = (size_t)ny * nz;
    mask.assign((size_t)nx * plane, 0);
    for (int x = 1; x < nx - 1; ++x)
        for (size_t p = 0; p < plane; ++p) {
            long v;
            if (!(f >> v)) { err = "geometry file " + file + " ends before " + std::to_string((size_t)(nx - 2) * plane) + " values"; return false; }
            if (v < 0 || v > 255) { err = "material number out of range in " + file; return false; }
            mask[(size_t)x * plane + p] = (uint8_t)v;
        }
    std::memcpy(&mask[0], &mask[plane], plane);
    std::memcpy(&mask[(size_t)(nx - 1) * plane], &mask[(size_t)(nx - 2) * plane], plane);
    return true;
}

bool write_fields(cl_ctx* h, const HostRun& run, long iT, std::vector<std::string>& index) {
    const cl_config& c = run.cfg;
    const size_t N = (size_t)c.nx * c.ny * c.nz;
    std::vector<double> buf(N);
    auto dump = [&](int field, int idx, const std::string& name) {
        if (!check(cl_get_field(h, field, idx, buf.data()), "cl_get_field")) return false;
        const std::string fn = name + "_" + std::to_string(iT) + ".raw";
        std::ofstream o(run.output_dir + "/" + fn, std::ios::binary);
        o.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)(N * sizeof(double)));
        index.push_back(fn);
        return (bool)o;
    };
    // the reference's VTI files (writeAdvVTI, writeNsVTI) beside the raw arrays
    std::string err;
    auto vti = [&](const std::string& prefix, std::vector<clhost::VtiArray> arrays) {
        const std::string fn = clhost::vti_name(prefix, iT);
        if (!clhost::write_vti(run.output_dir + "/" + fn, c.nx, c.ny, c.nz, arrays, err)) {
            std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
            return false;
        }
        index.push_back(fn);
        return true;
    };
    for (int s = 0; s < c.n_solutes; ++s) {
        if (!dump(CL_FIELD_CONC, s, run.subs_names[s])) return false;
        if (!vti(run.subs_names[s] + "_", {{"Density", 1, true, buf}})) return false;
    }
    for (int m = 0; m < c.n_microbes; ++m) {
        if (c.microbe_carrier[m]) continue;      // written as its carrier solute
        if (!dump(CL_FIELD_BIOMASS, m, run.microbe_names[m])) return false;
        if (!vti(run.microbe_names[m] + "_", {{"Density", 1, true, buf}})) return false;
    }
    // the material numbers (uint8), which precipitation and dissolution change
    std::vector<uint8_t> mask(N);
    if (!check(cl_download_mask(h, mask.data()), "cl_download_mask")) return false;
    const std::string fn = "mask_" + std::to_string(iT) + ".u8";
    std::ofstream o(run.output_dir + "/" + fn, std::ios::binary);
    o.write(reinterpret_cast<const char*>(mask.data()), (std::streamsize)N);
    index.push_back(fn);
    if (!o) return false;
    if (!vti(run.mask_filename + "_", {{"Density", 1, true, std::vector<double>(mask.begin(), mask.end())}}))
        return false;
    if (run.Pe > kThrd) {
        std::vector<double> u(3 * N), norm(N);
        for (int k = 0; k < 3; ++k)
            if (!check(cl_get_field(h, CL_FIELD_FLOW_U, k, u.data() + (size_t)k * N), "cl_get_field")) return false;
        for (size_t n = 0; n < N; ++n)
            norm[n] = std::sqrt(u[n] * u[n] + u[N + n] * u[N + n] + u[2 * N + n] * u[2 * N + n]);
        if (!vti("nsLattice_", {{"velocityNorm", 1, false, norm}, {"velocity", 3, false, u}})) return false;
    }
    return true;
}

// the configuration as raw cl_config bytes and the geometry as read
bool dump_config(const std::string& path, const cl_config& c, const std::vector<uint8_t>& mask) {
    std::ofstream o(path, std::ios::binary), om(path + ".mask", std::ios::binary);
    o.write(reinterpret_cast<const char*>(&c), (std::streamsize)sizeof c);
    om.write(reinterpret_cast<const char*>(mask.data()), (std::streamsize)mask.size());
    if (!o || !om) std::fprintf(stderr, "complab_b200: cannot write %s\n", path.c_str());
    return (bool)o && (bool)om;
}

// collideAndStream until the ValueTracer converges (cl_flow_solve); then the
// velocity statistics the calibration uses
bool flow_solve(cl_ctx* h, long max_it, double eps, int* iters) {
    const int st = cl_flow_solve(h, (int32_t)max_it, eps, iters);
    return check(st, "cl_flow_solve");
}

// PoreMeanU of the first solve with sessile microbes (complab.cpp:625-640):
// each pore material adds its masked mean velocity norm times its site count;
// each biofilm microbe adds the masked mean of its first material times the
// site count of all its materials; the sum is divided by the total count.  A
// material with no sites adds nothing (its masked mean would be 0/0).
bool weighted_pore_mean(cl_ctx* h, const cl_config& c, const HostRun& run, double* out) {
    double vel = 0.0;
    int64_t total = 0;
    auto masked = [&](int code, double* sum, int64_t* cnt) {
        return check(cl_flow_velocity_norm_masked(h, code, sum, cnt), "cl_flow_velocity_norm_masked");
    };
    for (int i = 0; i < c.n_pore_codes; ++i) {
        double su; int64_t n;
        if (!masked(c.pore_codes[i], &su, &n)) return false;
        total += n;
        vel += su;
    }
    for (const auto& mats : run.bio_materials) {
        if (mats.empty()) continue;
        int64_t film = 0;
        double su0 = 0.0; int64_t n0 = 0;
        for (size_t k = 0; k < mats.size(); ++k) {
            double su; int64_t n;
            if (!masked(mats[k], &su, &n)) return false;
            film += n;
            if (k == 0) { su0 = su; n0 = n; }
        }
        total += film;
        if (n0 > 0) vel += su0 / (double)n0 * (double)film;
    }
    if (total > 0) *out = vel / (double)total;
    return true;
}


// A surrogate network file (the weights the reference compiles in with
// surrogateModel.hh): whitespace-separated keyed lists, '#' comments:
//   layers L   widths w0 .. wL   W0 (w1 x w0, row-major) b0 (w1) ... W{L-1} b{L-1}
//   x_offset, x_gain (w0 each), x_ymin, y_offset, y_gain (wL each), y_ymin,
//   optionally x_lo, x_hi (the input clamp box, w0 each)
bool read_surrogate_net(const std::string& path, cl_surrogate_net& net, std::string& err) {
    std::ifstream f(path);
    if (!f) { err = "cannot open " + path; return false; }
    std::map<std::string, std::vector<double>> kv;
    std::string line, key;
    while (std::getline(f, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        std::istringstream is(line);
        std::string tok;
        while (is >> tok) {
            char* end = nullptr;
            const double v = std::strtod(tok.c_str(), &end);
            if (end && *end == '\0' && !key.empty()) kv[key].push_back(v);
            else key = tok;
        }
    }
    auto need = [&](const std::string& k, size_t n) -> const std::vector<double>* {
        auto it = kv.find(k);
        if (it == kv.end() || it->second.size() != n) { err = path + ": " + k + " needs " + std::to_string(n) + " numbers"; return nullptr; }
        return &it->second;
    };
    net = cl_surrogate_net{};
    const auto* L = need("layers", 1);
    if (!L) return false;
    net.n_layers = (int32_t)(*L)[0];
    if (net.n_layers < 1 || net.n_layers > CL_SRG_MAX_LAYERS) { err = path + ": 1.." + std::to_string(CL_SRG_MAX_LAYERS) + " layers"; return false; }
    const auto* W = need("widths", (size_t)net.n_layers + 1);
    if (!W) return false;
    for (int l = 0; l <= net.n_layers; ++l) {
        net.widths[l] = (int32_t)(*W)[l];
        if (net.widths[l] < 1 || net.widths[l] > CL_SRG_MAX_WIDTH) { err = path + ": widths 1.." + std::to_string(CL_SRG_MAX_WIDTH); return false; }
    }
    size_t off = 0;
    for (int l = 0; l < net.n_layers; ++l) {
        const size_t wi = net.widths[l], wo = net.widths[l + 1];
        const auto* w = need("W" + std::to_string(l), wi * wo);
        const auto* b = need("b" + std::to_string(l), wo);
        if (!w || !b) return false;
        if (off + wi * wo + wo > 4096) { err = path + ": too many parameters"; return false; }
        for (size_t k = 0; k < wi * wo; ++k) net.params[off++] = (*w)[k];
        for (size_t k = 0; k < wo; ++k) net.params[off++] = (*b)[k];
    }
    const size_t w0 = net.widths[0], wl = net.widths[net.n_layers];
    const auto *xo = need("x_offset", w0), *xg = need("x_gain", w0), *xy = need("x_ymin", 1);
    const auto *yo = need("y_offset", wl), *yg = need("y_gain", wl), *yy = need("y_ymin", 1);
    if (!xo || !xg || !xy || !yo || !yg || !yy) return false;
    for (size_t k = 0; k < w0; ++k) {
        net.x_offset[k] = (*xo)[k]; net.x_gain[k] = (*xg)[k];
        net.x_lo[k] = kv.count("x_lo") && kv["x_lo"].size() == w0 ? kv["x_lo"][k] : -1e308;
        net.x_hi[k] = kv.count("x_hi") && kv["x_hi"].size() == w0 ? kv["x_hi"][k] : 1e308;
    }
    for (size_t k = 0; k < wl; ++k) { net.y_offset[k] = (*yo)[k]; net.y_gain[k] = (*yg)[k]; }
    net.x_ymin = (*xy)[0];
    net.y_ymin = (*yy)[0];
    return true;
}

}  // namespace

int main(int argc, char** argv) {
    std::string xml = "CompLaB.xml", rates, dump, restart;
    std::vector<std::string> srg_files;
    long steps_override = -1;
    int eq_solver = -1;
    bool print_config = false, quiet = false;
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--print-config") print_config = true;
        else if (a == "--quiet") quiet = true;
        else if (a == "--steps" && i + 1 < argc) steps_override = std::atol(argv[++i]);
        else if (a == "--rates" && i + 1 < argc) rates = argv[++i];
        else if (a == "--surrogate" && i + 1 < argc) srg_files.push_back(argv[++i]);
        else if (a == "--dump-config" && i + 1 < argc) dump = argv[++i];
        else if (a == "--restart" && i + 1 < argc) restart = argv[++i];
        else if (a == "--eq-solver" && i + 1 < argc && (std::strcmp(argv[i + 1], "pcf") == 0 ||
                                                         std::strcmp(argv[i + 1], "newton") == 0))
            eq_solver = std::strcmp(argv[++i], "pcf") == 0 ? CL_EQ_SOLVER_PCF : CL_EQ_SOLVER_NEWTON;
        else if (!a.empty() && a[0] != '-') xml = a;
        else {
            std::fprintf(stderr, "usage: %s [CompLaB.xml] [--steps N] [--eq-solver newton|pcf] [--rates rates.xml] "
                         "[--surrogate net.txt]... [--restart DIR] [--dump-config FILE] [--print-config] [--quiet]\n",
                         argv[0]);
            return 2;
        }
    }
    HostRun run;
    std::string err;
    if (clhost::read_complab_xml(xml, run, err, rates)) { std::fprintf(stderr, "complab_b200: %s\n", err.c_str()); return 1; }
    if (eq_solver >= 0) run.cfg.eq.solver = eq_solver;
    run.srg_files = srg_files;
    // each surrogate organism's network: its inputs are the Fin of the first
    // solutes in order (the shipped model reads Fin[m][0], Fin[m][1]), its
    // first output the growth rate, further outputs the Fout of the solutes
    std::vector<cl_surrogate_net> nets(run.cfg.n_srg);
    if ((int)srg_files.size() < run.cfg.n_srg) {
        std::fprintf(stderr, "complab_b200: %d surrogate organism(s) need a network each (--surrogate FILE)\n", run.cfg.n_srg);
        return 1;
    }
    for (int o = 0; o < run.cfg.n_srg; ++o) {
        if (!read_surrogate_net(srg_files[o], nets[o], err)) { std::fprintf(stderr, "complab_b200: %s\n", err.c_str()); return 1; }
        cl_srg_organism& g = run.cfg.srg[o];
        const int w0 = nets[o].widths[0], wl = nets[o].widths[nets[o].n_layers];
        if (w0 > run.cfg.n_solutes || wl - 1 > run.cfg.n_solutes) {
            std::fprintf(stderr, "complab_b200: network %s: more inputs or outputs than solutes\n", srg_files[o].c_str());
            return 1;
        }
        for (int k = 0; k < w0; ++k) { g.in_kind[k] = CL_SRG_IN_FIN; g.in_index[k] = k; }
        g.out_kind[0] = CL_SRG_OUT_GROWTH; g.out_index[0] = 0;
        for (int q = 1; q < wl; ++q) { g.out_kind[q] = CL_SRG_OUT_FOUT; g.out_index[q] = q - 1; }
    }
    if (print_config && dump.empty()) { std::printf("%s\n", clhost::run_json(run).c_str()); return 0; }
    if (steps_override >= 0) run.ade_max = steps_override;
    if (!print_config)
        for (const std::string& n : run.notes) if (!quiet) std::fprintf(stderr, "complab_b200: note: %s\n", n.c_str());

    cl_config& c = run.cfg;
    std::vector<uint8_t> mask;
    if (!read_geometry(run.input_dir + "/" + run.geom_file, c.nx, c.ny, c.nz, mask, err)) {
        std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
        return 1;
    }
    // with --print-config, the dump is the configuration as parsed (before
    // any flow calibration) and needs no GPU
    if (print_config) {
        std::printf("%s\n", clhost::run_json(run).c_str());
        return dump_config(dump, c, mask) ? 0 : 1;
    }
    // a restart takes the geometry (as it was when saved), the calibrated
    // pressure, dt and relaxation from the checkpoint
    clhost::Checkpoint chk;
    if (!restart.empty()) {
        if (!clhost::read_checkpoint(restart, run, chk, mask, err)) {
            std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
            return 1;
        }
        c.rho_in = chk.rho_in;
        c.rho_out = chk.rho_out;
        c.dt = chk.dt;
        run.delta_P = chk.delta_P;
        for (int s = 0; s < c.n_solutes; ++s) { c.omega_pore[s] = chk.omega_pore[s]; c.omega_bio[s] = chk.omega_bio[s]; }
    }
    const auto t0 = std::chrono::steady_clock::now();
    int st = 0;
    Ctx ctx;
    ctx.h = cl_create(&c, nullptr, &st);
    if (!ctx.h) { std::fprintf(stderr, "complab_b200: cl_create failed (%d): %s\n", st, cl_last_error()); return 1; }
    cl_ctx* h = ctx.h;
    for (int o = 0; o < c.n_srg; ++o)
        if (!check(cl_set_surrogate(h, o, &nets[o]), "cl_set_surrogate")) return 1;
    if (!check(cl_upload_mask(h, mask.data()), "cl_upload_mask")) return 1;
    if (!restart.empty() && !clhost::restore_dynamics(h, run, restart, err)) {
        std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
        return 1;
    }

    // flow and the Peclet calibration
    const double nsNu = (run.tau - 0.5) / 3.0;
    double pore_mean_u = 0.0, max_ux = 0.0, outlet_ux = 0.0, pe_achieved = 0.0;
    int ns_iters = 0;
    if (!check(cl_flow_init(h), "cl_flow_init")) return 1;
    if (!restart.empty() && chk.has_flow && !clhost::restore_flow(h, run, restart, err)) {
        std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
        return 1;
    }
    if (run.Pe > kThrd && restart.empty()) {
        if (!flow_solve(h, run.ns_max1, run.ns_conv1, &ns_iters)) return 1;
        if (!check(cl_flow_velocity_stats(h, &pore_mean_u, &max_ux, &outlet_ux), "cl_flow_velocity_stats")) return 1;
        // with sessile microbes the first solve's pore mean is the count-weighted
        // mean over the pore materials and each microbe's biofilm materials, the
        // biofilm taking the mean of its first material (complab.cpp:625-640)
        bool sessile = false;
        for (const auto& mats : run.bio_materials) sessile = sessile || !mats.empty();
        if (sessile && !weighted_pore_mean(h, c, run, &pore_mean_u)) return 1;
        const double D_fixed = 0.25 * (0.8 - 0.5);          // tau_ADE_fixed = 0.8 (complab.cpp:164)
        const double perm = outlet_ux * nsNu * run.charcs_length / run.delta_P;
        const double u_target = run.Pe * D_fixed / run.charcs_length;
        const double dP_new = u_target * nsNu * run.charcs_length / perm;
        if (std::fabs(dP_new - run.delta_P) / run.delta_P > 0.01) {
            run.delta_P = dP_new;
            if (!check(cl_set_flow_pressure(h, 1.0, 1.0 - 3.0 * dP_new), "cl_set_flow_pressure")) return 1;
            c.rho_in = 1.0;
            c.rho_out = 1.0 - 3.0 * dP_new;
            if (!check(cl_flow_init(h), "cl_flow_init")) return 1;
            if (!flow_solve(h, run.ns_max1, run.ns_conv1, &ns_iters)) return 1;
            if (!check(cl_flow_velocity_stats(h, &pore_mean_u, &max_ux, &outlet_ux), "cl_flow_velocity_stats")) return 1;
        }
        pe_achieved = outlet_ux * run.charcs_length / D_fixed;
        // performStabilityChecks (complab.cpp:77-93, 673-686): Ma = u_max / sqrt(1/3)
        // and CFL = u_max below 1, tau_NS in (0.5, 2); warnings for Ma > 0.3 and
        // a grid Peclet number u_max / D above 2
        const double Ma = max_ux / std::sqrt(1.0 / 3.0), Pe_grid = D_fixed > kThrd ? max_ux / D_fixed : 0.0;
        if (!(Ma < 1.0) || !(max_ux < 1.0) || !(run.tau > 0.5 && run.tau < 2.0)) {
            std::fprintf(stderr, "complab_b200: stability check failed before the run (Ma %g, CFL %g, tau_NS %g): "
                                 "lower deltaP or Pe, or adjust tau\n", Ma, max_ux, run.tau);
            return 1;
        }
        if (Ma > 0.3) std::fprintf(stderr, "complab_b200: warning: Ma=%g > 0.3 (flow re-solves may diverge)\n", Ma);
        if (!(Pe_grid < 2.0))
            std::fprintf(stderr, "complab_b200: warning: Pe_grid=%g > 2 (advection may overshoot into negatives)\n", Pe_grid);
    }

    // solute relaxation and dt from the flow (complab.cpp:708-727)
    const int S = c.n_solutes;
    if (S > 0 && !restart.empty()) {
        if (!check(cl_set_transport(h, c.omega_pore, c.omega_bio, c.dt), "cl_set_transport")) return 1;
    } else if (S > 0) {
        double refNu, refTau;
        if (run.Pe > kThrd) {
            refNu = pore_mean_u * run.charcs_length / run.Pe;
            refTau = refNu * 4.0 + 0.5;
            if (refTau > 2 || refTau <= 0.5) { std::fprintf(stderr, "complab_b200: transport tau=%g invalid\n", refTau); return 1; }
        } else {
            refTau = run.tau;
            refNu = 0.25 * (refTau - 0.5);
        }
        std::vector<double> om_p(S), om_b(S);
        for (int s = 0; s < S; ++s) {
            const double nu = refNu * run.D_pore[s] / run.D_pore[0];
            om_p[s] = 1.0 / (nu * 4.0 + 0.5);
            om_b[s] = 1.0 / (refNu * run.D_bfilm[s] / run.D_bfilm_ref[s] * 4.0 + 0.5);
        }
        const double dt = refNu * run.dx * run.dx / run.D_pore[0];
        c.dt = dt;
        for (int s = 0; s < S; ++s) { c.omega_pore[s] = om_p[s]; c.omega_bio[s] = om_b[s]; }
        if (!check(cl_set_transport(h, om_p.data(), om_b.data(), dt), "cl_set_transport")) return 1;
    }
    if (run.Pe > kThrd && !check(cl_couple_velocity(h), "cl_couple_velocity")) return 1;
    if (!check(cl_ade_init(h), "cl_ade_init")) return 1;
    if (!dump.empty() && !dump_config(dump, c, mask)) return 1;
    if (!restart.empty() && !clhost::restore_transport(h, run, restart, err)) {
        std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
        return 1;
    }
    // sessile biomass on the microbes' materials (initializeScalarLattice3D)
    if (restart.empty()) {
        const size_t N = mask.size();
        std::vector<double> b(N);
        for (int m = 0; m < c.n_microbes; ++m) {
            if (c.microbe_carrier[m]) continue;      // an LBM-solved microbe starts as its carrier's c0
            std::fill(b.begin(), b.end(), 0.0);
            const auto& mats = run.bio_materials[m];
            const auto& b0 = run.b0[m];
            for (size_t n = 0; n < N; ++n)
                for (size_t k = 0; k < mats.size() && k < b0.size(); ++k)
                    if (mask[n] == mats[k]) b[n] = b0[k];
            if (!check(cl_set_field(h, CL_FIELD_BIOMASS, m, b.data()), "cl_set_field")) return 1;
        }
    }

    long resolves = 0, ca_sweeps = 0, ca_blocks = 0, ca_changes = 0;
    // finite-difference microbes and their nu = bioNUinPore[0] (refNu from the
    // first solute's pore relaxation, complab.cpp:716-736)
    uint32_t fd_bits = 0;
    for (int m = 0; m < c.n_microbes && m < 32; ++m) if (m < (int)run.fd.size() && run.fd[m]) fd_bits |= 1u << m;
    const double fd_nu = c.n_solutes > 0 ? (1.0 / c.omega_pore[0] - 0.5) / 4.0 * fd_nu_ratio(run) : 0.0;
    if (c.ca_enabled) {
        // initial mask update from the seeded biomass, and on a change the
        // dynamics switch and a flow re-solve (complab.cpp:1068-1091)
        int64_t ch = 0;
        if (!check(cl_ca_update_mask(h, &ch), "cl_ca_update_mask")) return 1;
        ca_changes += ch;
        if (ch > 0) {
            if (!check(cl_update_dynamics(h), "cl_update_dynamics")) return 1;
            if (run.Pe > kThrd) {
                int it2 = 0;
                if (!check(cl_flow_solve(h, (int32_t)run.ns_max1, run.ns_conv1, &it2), "cl_flow_solve")) return 1;
                if (!check(cl_couple_velocity(h), "cl_couple_velocity")) return 1;
                ++resolves;
            }
        }
    }

    mkdir(run.output_dir.c_str(), 0777);
    std::vector<std::string> index;
    long nonconv_steps = 0, precip_changes = 0, dissol_changes = 0, steps_done = 0;
    const char* stopped = "";
    const auto t1 = std::chrono::steady_clock::now();
    for (long iT = restart.empty() ? 0 : chk.steps; iT < run.ade_max; ++iT) {
        st = cl_step(h, 1);
        if (!check(st, "cl_step")) return 1;
        ++steps_done;
        if (st == CL_WARN_NOT_CONVERGED) ++nonconv_steps;
        // CA biomass redistribution (complab.cpp:1453-1715), or the
        // finite-difference step of sessile biomass: the mask update, one
        // diffusion step, the mask update (complab.cpp:1716-1731)
        bool ca_changed = false;
        if (c.ca_enabled && fd_bits) {
            int64_t ch1 = 0, ch2 = 0;
            if (!check(cl_ca_update_mask(h, &ch1), "cl_ca_update_mask")) return 1;
            if (!check(cl_fd_diffuse(h, fd_nu, fd_bits), "cl_fd_diffuse")) return 1;
            if (!check(cl_ca_update_mask(h, &ch2), "cl_ca_update_mask")) return 1;
            ca_changes += ch1 + ch2;
            ca_changed = ch1 + ch2 > 0;
        } else if (c.ca_enabled) {
            int32_t sw = 0;
            int64_t ch = 0;
            double bm = 0.0;
            st = cl_ca_redistribute(h, &sw, &ch, &bm);
            if (!check(st, "cl_ca_redistribute")) return 1;
            ca_sweeps += sw;
            ca_blocks += sw > 0;
            ca_changes += ch;
            ca_changed = ch > 0;
            if (st == CL_WARN_NOT_CONVERGED) {
                // the reference writes every field and ends the run here
                std::fprintf(stderr, "complab_b200: CA redistribution did not settle at iT=%ld (max biomass %g)\n", iT, bm);
                stopped = "ca_not_settled";
                if (!write_fields(h, run, iT, index)) return 1;
                break;
            }
        }
        bool changed = false;
        if (c.precip_enabled && iT % run.precip_interval == 0) {
            int64_t ch = 0;
            if (!check(cl_precip_convert(h, &ch), "cl_precip_convert")) return 1;
            precip_changes += ch;
            changed = changed || ch > 0;
        }
        if (c.dissol_enabled && iT % run.dissol_interval == 0) {
            int64_t ch = 0;
            if (!check(cl_dissol_convert(h, &ch), "cl_dissol_convert")) return 1;
            dissol_changes += ch;
            changed = changed || ch > 0;
        }
        // a CA mask change switches the dynamics on ade_update_interval and
        // re-solves the flow on ns_update_interval (complab.cpp:1734-1780)
        const bool ca_dyn = ca_changed && (iT % run.ade_update_interval == 0 || iT % run.ns_update_interval == 0);
        const bool ca_ns = ca_changed && iT % run.ns_update_interval == 0;
        if ((changed && run.Pe > kThrd) || ca_dyn) {
            if (!check(cl_update_dynamics(h), "cl_update_dynamics")) return 1;
        }
        if (run.Pe > kThrd && (changed || ca_ns)) {
            int it2 = 0;
            st = cl_flow_solve(h, (int32_t)run.ns_max2, run.ns_conv2, &it2);
            if (!check(st, "cl_flow_solve")) return 1;
            if (!check(cl_couple_velocity(h), "cl_couple_velocity")) return 1;
            ++resolves;
        }
        if (run.vtk_interval > 0 && iT % run.vtk_interval == 0 && !write_fields(h, run, iT, index)) return 1;
        // checkpoint of the state after iT + 1 steps (the reference's save_CHK_interval)
        if (run.chk_interval > 0 && (iT + 1) % run.chk_interval == 0) {
            clhost::Checkpoint now;
            now.steps = iT + 1;
            now.rho_in = c.rho_in;
            now.rho_out = c.rho_out;
            now.dt = c.dt;
            now.delta_P = run.delta_P;
            now.omega_pore.assign(c.omega_pore, c.omega_pore + c.n_solutes);
            now.omega_bio.assign(c.omega_bio, c.omega_bio + c.n_solutes);
            now.has_flow = run.Pe > kThrd;
            const std::string dir = run.output_dir + "/chk_" + std::to_string(iT + 1);
            if (!clhost::save_checkpoint(h, run, now, dir, err)) {
                std::fprintf(stderr, "complab_b200: %s\n", err.c_str());
                return 1;
            }
        }
    }
    const auto t2 = std::chrono::steady_clock::now();
    if (!*stopped && !write_fields(h, run, run.ade_max, index)) return 1;
    {
        std::ofstream o(run.output_dir + "/fields.json");
        o << "{\"nx\": " << c.nx << ", \"ny\": " << c.ny << ", \"nz\": " << c.nz
          << ", \"dtype\": \"float64\", \"order\": \"(x*ny + y)*nz + z\", \"files\": [";
        for (size_t i = 0; i < index.size(); ++i) o << (i ? ", " : "") << "\"" << index[i] << "\"";
        o << "]}\n";
    }
    const double setup_s = std::chrono::duration<double>(t1 - t0).count();
    const double loop_s = std::chrono::duration<double>(t2 - t1).count();
    const double sites = (double)mask.size();
    std::printf("{\"steps\": %ld, \"setup_s\": %.6f, \"loop_s\": %.6f, \"mlups\": %.3f, \"ns_iters\": %d, "
                "\"pore_mean_u\": %.9g, \"max_ux\": %.9g, \"outlet_ux\": %.9g, \"delta_P\": %.9g, \"Pe_achieved\": %.6g, "
                "\"dt\": %.9g, \"nonconverged_steps\": %ld, \"precip_changes\": %lld, \"dissol_changes\": %lld, "
                "\"ca_sweeps\": %ld, \"ca_blocks\": %ld, \"ca_mask_changes\": %ld, "
                "\"flow_resolves\": %ld, \"stopped\": \"%s\", \"output\": \"%s\"}\n",
                steps_done, setup_s, loop_s, loop_s > 0 ? sites * steps_done / loop_s / 1e6 : 0.0, ns_iters,
                pore_mean_u, max_ux, outlet_ux, run.delta_P, pe_achieved, c.dt, nonconv_steps,
                (long long)precip_changes, (long long)dissol_changes, ca_sweeps, ca_blocks, ca_changes,
                resolves, stopped, run.output_dir.c_str());
    return *stopped ? 3 : 0;
}
