// complab_xml.cpp -- CompLaB.xml -> cl_config (see complab_xml.h).
#include "complab_xml.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>

#include "xml_lite.h"

namespace clhost {

namespace {

constexpr double kThrd = 1e-12;    // COMPLAB_THRD

std::string lower(std::string s) {
    for (auto& c : s) c = (char)std::tolower((unsigned char)c);
    return s;
}

const XmlNode* opt(const XmlNode& n, std::initializer_list<const char*> path) {
    const XmlNode* p = &n;
    for (const char* k : path) {
        p = p->find(k);
        if (!p) return nullptr;
    }
    return p;
}

double num_or(const XmlNode& n, std::initializer_list<const char*> path, double dflt) {
    const XmlNode* p = opt(n, path);
    return p ? p->num() : dflt;
}

// "s:v s:v ..." pairs (solute index : value)
std::vector<std::pair<int, double>> pairs(const XmlNode& n) {
    std::vector<std::pair<int, double>> out;
    for (const std::string& w : n.words()) {
        const size_t c = w.find(':');
        if (c == std::string::npos) throw std::runtime_error("expected index:value in " + n.path + ", got " + w);
        out.emplace_back(std::stoi(w.substr(0, c)), std::stod(w.substr(c + 1)));
    }
    return out;
}

int bc_type(const XmlNode& n) {
    const std::string t = lower(n.str());
    if (t == "dirichlet") return CL_BC_DIRICHLET;
    if (t == "neumann") return CL_BC_NEUMANN;
    throw std::runtime_error(n.path + " (" + n.str() + ") should be either Dirichlet or Neumann");
}

}  // namespace

int read_complab_xml(const std::string& path, HostRun& run, std::string& err, const std::string& rates) {
    try {
        XmlDoc doc(path);
        const XmlNode& P = doc["parameters"];
        // the rate-law blocks the main file lacks come from the rates file
        std::unique_ptr<XmlDoc> rdoc;
        if (!rates.empty()) rdoc = std::make_unique<XmlDoc>(rates);
        const XmlNode* RP = rdoc ? &(*rdoc)["parameters"] : nullptr;
        cl_config& c = run.cfg;
        std::memset(&c, 0, sizeof c);
        const size_t slash = path.find_last_of('/');
        run.xml_dir = slash == std::string::npos ? "." : path.substr(0, slash);

        // simulation mode (complab_functions.hh:653-735)
        bool enable_kinetics = true, enable_abiotic = false;
        if (const XmlNode* m = opt(P, {"simulation_mode"})) {
            if (const XmlNode* v = m->find("biotic_mode")) {
                const std::string t = lower(v->str());
                run.biotic_mode = !(t == "no" || t == "false" || t == "0" || t == "abiotic");
            }
            if (const XmlNode* v = m->find("enable_kinetics")) {
                const std::string t = lower(v->str());
                enable_kinetics = !(t == "no" || t == "false" || t == "0");
            }
            if (const XmlNode* v = m->find("enable_abiotic_kinetics")) enable_abiotic = v->flag();
            if (const XmlNode* v = m->find("enable_surrogate")) run.enable_surrogate = v->flag();
            if (const XmlNode* v = m->find("enable_fba_glpk"); v && v->flag())
                run.notes.push_back("FBA (GLPK) reaction type is not part of this library; ignored");
            if (const XmlNode* v = m->find("enable_fba_cobrapy"); v && v->flag())
                run.notes.push_back("FBA (COBRApy) reaction type is not part of this library; ignored");
        }
        if (!run.biotic_mode) enable_kinetics = false;

        // required inputs (complab_functions.hh:767-800)
        const XmlNode& dom = P["LB_numerics"]["domain"];
        c.nx = (int32_t)dom["nx"].integer() + 2;
        c.ny = (int32_t)dom["ny"].integer();
        c.nz = (int32_t)dom["nz"].integer();
        double dx = dom["dx"].num();
        run.geom_file = dom["filename"].str();
        const XmlNode& chem = P["chemistry"];
        int S = (int)chem["number_of_substrates"].integer();
        if (S < 0 || S > CL_MAX_SOLUTES) throw std::runtime_error("number_of_substrates out of range");
        c.n_solutes = S;
        for (int s = 0; s < S; ++s) {
            const XmlNode& sub = chem["substrate" + std::to_string(s)];
            c.left_type[s] = bc_type(sub["left_boundary_type"]);
            c.right_type[s] = bc_type(sub["right_boundary_type"]);
            c.left_value[s] = sub["left_boundary_condition"].num();
            c.right_value[s] = sub["right_boundary_condition"].num();
        }

        // microbiology: CA- or finite-difference-solved sessile biomass, or
        // LBM-solved biomass carried by an extra mobile solute (a planktonic
        // bFree lattice, complab.cpp:788-797)
        int M = 0;
        if (run.biotic_mode) {
            const XmlNode& mic = P["microbiology"];
            M = (int)mic["number_of_microbes"].integer();
            if (M < 0 || M > CL_MAX_MICROBES) throw std::runtime_error("number_of_microbes out of range");
            for (int m = 0; m < M; ++m) {
                const XmlNode& mb = mic["microbe" + std::to_string(m)];
                const std::string st = lower(mb["solver_type"].str());
                const bool fd = st == "fd" || st == "finite difference" || st == "finite_difference";
                // the biomass pore diffusion coefficient, which finite differences need
                // (complab_functions.hh:1123-1130); microbe 0's sets their nu
                const XmlNode* dpo = opt(mb, {"biomass_diffusion_coefficients", "in_pore"});
                if (fd && !dpo)
                    throw std::runtime_error("microbe" + std::to_string(m) +
                                             ": biomass_diffusion_coefficients must be defined when solver_type is Finite Difference");
                if (m == 0 && dpo) run.D_bmass_pore0 = dpo->num();
                run.fd.push_back(fd ? 1 : 0);
                // the surrogate reaction type (run_surrogate3D with MetabolicConfig,
                // complab3d_metabolic.hh:772-800): Vmax from <fba_maximum_uptake_flux>,
                // else <maximum_uptake_flux>; Kc from <half_saturation_constants>;
                // <biomass_molar_mass> (24.6 gDW/mol by default); kd the decay
                const std::string rt = mb.has("reaction_type") ? lower(mb["reaction_type"].str()) : "";
                if (run.enable_surrogate && rt.find("surrogate") != std::string::npos) {
                    if (c.n_srg >= CL_MAX_SRG_ORG) throw std::runtime_error("more surrogate organisms than the library holds");
                    cl_srg_organism& g = c.srg[c.n_srg];
                    g.microbe = m;
                    g.net = c.n_srg;
                    const XmlNode* vm = opt(mb, {"fba_maximum_uptake_flux"});
                    if (!vm) vm = opt(mb, {"maximum_uptake_flux"});
                    if (!vm) throw std::runtime_error("microbe" + std::to_string(m) + ": the surrogate needs <fba_maximum_uptake_flux>");
                    const std::vector<double> vmax = vm->nums();
                    const std::vector<double> kc = mb.has("half_saturation_constants") ? mb["half_saturation_constants"].nums()
                                                                                       : std::vector<double>();
                    for (int s = 0; s < CL_MAX_SOLUTES; ++s) {
                        g.vmax[s] = s < (int)vmax.size() ? std::fabs(vmax[s]) : 0.0;
                        g.kc[s] = s < (int)kc.size() ? kc[s] : 0.0;
                    }
                    g.mw = num_or(mb, {"biomass_molar_mass"}, 24.6);
                    g.kd = num_or(mb, {"decay_coefficient"}, 0.0);
                    ++c.n_srg;
                }
                run.carried.push_back(st == "lbm" || st == "lb" || st == "lattice boltzmann" ? 1 : 0);
                run.b0.push_back(mb["initial_densities"].nums());
                run.microbe_names.push_back(mb.has("name_of_microbes") ? mb["name_of_microbes"].str()
                                                                       : "microbe" + std::to_string(m));
                c.decay[m] = num_or(mb, {"decay_coefficient"}, 0.0);
            }
        }
        c.n_microbes = M;

        // paths (defaults src / input / output)
        auto path_or = [&](const char* k, const char* d) {
            const XmlNode* p = opt(P, {"path", k});
            return p ? p->str() : std::string(d);
        };
        run.input_dir = run.xml_dir + "/" + path_or("input_path", "input");
        run.output_dir = run.xml_dir + "/" + path_or("output_path", "output");

        // LB numerics with defaults (complab_functions.hh:948-1030)
        run.delta_P = num_or(P, {"LB_numerics", "delta_P"}, 0.0);
        run.Pe = num_or(P, {"LB_numerics", "Peclet"}, 0.0);
        if (run.delta_P < kThrd) run.Pe = 0.0;
        run.tau = num_or(P, {"LB_numerics", "tau"}, 0.8);
        run.charcs_length = num_or(dom, {"characteristic_length"}, 0.0);
        const std::string unit = dom.has("unit") ? dom["unit"].str() : std::string("um");
        run.charcs_length /= dx;
        if (unit == "mm") dx *= 1e-3;
        else if (unit == "um") dx *= 1e-6;        // also the default when <unit> is absent
        run.dx = dx;
        const XmlNode* mat = opt(dom, {"material_numbers"});
        std::vector<double> pore = mat && mat->has("pore") ? (*mat)["pore"].nums() : std::vector<double>{2.0};
        c.n_pore_codes = (int32_t)std::min<size_t>(pore.size(), CL_MAX_CODES);
        for (int i = 0; i < c.n_pore_codes; ++i) c.pore_codes[i] = (int32_t)pore[i];
        c.solid_code = mat && mat->has("solid") ? (int32_t)(*mat)["solid"].integer() : 0;
        c.bb_code = mat && mat->has("bounce_back") ? (int32_t)(*mat)["bounce_back"].integer() : 1;
        for (int m = 0; m < M; ++m) {
            std::vector<int> codes;
            if (mat && mat->has("microbe" + std::to_string(m)))
                for (double v : (*mat)["microbe" + std::to_string(m)].nums()) codes.push_back((int)v);
            run.bio_materials.push_back(codes);
            for (int v : codes)
                if (c.n_bio_codes < CL_MAX_CODES &&
                    std::find(c.bio_codes, c.bio_codes + c.n_bio_codes, v) == c.bio_codes + c.n_bio_codes)
                    c.bio_codes[c.n_bio_codes++] = v;
        }
        const XmlNode* it = opt(P, {"LB_numerics", "iteration"});
        if (it) {
            run.ns_max1 = (long)num_or(*it, {"ns_max_iT1"}, 100000);
            run.ns_max2 = (long)num_or(*it, {"ns_max_iT2"}, 100000);
            run.ns_conv1 = num_or(*it, {"ns_converge_iT1"}, 1e-8);
            run.ns_conv2 = num_or(*it, {"ns_converge_iT2"}, 1e-6);
            run.ade_max = (long)num_or(*it, {"ade_max_iT"}, 10000000);
            run.ns_update_interval = std::max(1L, (long)num_or(*it, {"ns_update_interval"}, 1));
            run.ade_update_interval = std::max(1L, (long)num_or(*it, {"ade_update_interval"}, 1));
        }
        run.vtk_interval = (long)num_or(P, {"IO", "save_VTK_interval"}, 0);
        run.chk_interval = (long)num_or(P, {"IO", "save_CHK_interval"}, 0);
        if (const XmlNode* mf = opt(P, {"IO", "mask_filename"})) run.mask_filename = mf->str();

        // substrates (complab_functions.hh:1031-1048; immobile complab.cpp:244-266)
        for (int s = 0; s < S; ++s) {
            const XmlNode& sub = chem["substrate" + std::to_string(s)];
            run.subs_names.push_back(sub.has("name_of_substrates") ? sub["name_of_substrates"].str()
                                                                   : "substrate_" + std::to_string(s));
            run.D_pore.push_back(num_or(sub, {"substrate_diffusion_coefficients", "in_pore"}, 1e-9));
            run.D_bfilm.push_back(num_or(sub, {"substrate_diffusion_coefficients", "in_biofilm"}, 2e-10));
            c.c0[s] = num_or(sub, {"initial_concentration"}, 0.0);
            c.immobile[s] = sub.has("immobile") && sub["immobile"].flag() ? 1 : 0;
            run.D_bfilm_ref.push_back(0.0);
        }
        for (int s = 0; s < S; ++s) run.D_bfilm_ref[s] = run.D_pore[0];
        // an LBM-solved microbe: one more mobile solute named after it, with
        // its diffusion, its boundaries and its initial density everywhere
        // (soluteDomainSetup with vec_b0_free, complab.cpp:791-792)
        for (int m = 0; m < M; ++m) {
            if (!run.carried[m]) continue;
            if (S >= CL_MAX_SOLUTES) throw std::runtime_error("too many solutes with the LBM-solved microbes");
            const XmlNode& mb = P["microbiology"]["microbe" + std::to_string(m)];
            const int s = S++;
            run.subs_names.push_back(run.microbe_names[m]);
            const double dp = num_or(mb, {"biomass_diffusion_coefficients", "in_pore"}, 0.0);
            run.D_pore.push_back(dp);
            run.D_bfilm.push_back(num_or(mb, {"biomass_diffusion_coefficients", "in_biofilm"}, 0.0));
            run.D_bfilm_ref.push_back(dp);
            c.c0[s] = run.b0[m].empty() ? 0.0 : run.b0[m][0];
            c.immobile[s] = 0;
            c.left_type[s] = mb.has("left_boundary_type") ? bc_type(mb["left_boundary_type"]) : CL_BC_NEUMANN;
            c.right_type[s] = mb.has("right_boundary_type") ? bc_type(mb["right_boundary_type"]) : CL_BC_NEUMANN;
            c.left_value[s] = num_or(mb, {"left_boundary_condition"}, 0.0);
            c.right_value[s] = num_or(mb, {"right_boundary_condition"}, 0.0);
            c.microbe_carrier[m] = s + 1;
        }
        c.n_solutes = S;
        if (enable_abiotic && S < 1) throw std::runtime_error("abiotic kinetics needs at least one substrate");

        // flow numbers; the solute relaxation and dt follow from the flow
        // (complab.cpp:708-727), so the driver sets them after the flow solve
        c.tau_ns = run.tau;
        c.rho_in = 1.0;
        c.rho_out = 1.0 - run.delta_P * 3.0;
        c.perm_ratio = 0.0;
        for (int m = 0; m < M; ++m) {
            const XmlNode& mb = P["microbiology"]["microbe" + std::to_string(m)];
            if (const XmlNode* v = mb.find("viscosity_ratio_in_biofilm")) {
                const double nu0 = v->num();
                if (m == 0) c.perm_ratio = nu0 > kThrd ? 1.0 / nu0 : 0.0;
            }
        }
        const double refTau = run.tau, refNu = 0.25 * (refTau - 0.5);
        for (int s = 0; s < S; ++s) {
            const double nu = refNu * run.D_pore[s] / run.D_pore[0];
            c.omega_pore[s] = 1.0 / (nu * 4.0 + 0.5);
            c.omega_bio[s] = 1.0 / (refNu * run.D_bfilm[s] / run.D_bfilm_ref[s] * 4.0 + 0.5);
        }
        c.dt = S > 0 ? refNu * dx * dx / run.D_pore[0] : 1.0;

        // rate laws: the table that stands for defineKinetics.hh /
        // defineAbioticKinetics.hh
        const XmlNode* rtab = opt(P, {"rate_table"});
        if (!rtab && RP) rtab = opt(*RP, {"rate_table"});
        if (const XmlNode* rt = rtab) {
            // <decay>m:kd ...</decay>: first-order decay that the compiled rate law
            // applies itself, in place of the microbe's <decay_coefficient>
            if (const XmlNode* dk = rt->find("decay"))
                for (auto& pv : pairs(*dk)) {
                    if (pv.first < 0 || pv.first >= M) throw std::runtime_error("decay microbe index out of range in " + dk->path);
                    c.decay[pv.first] = pv.second;
                }
            for (int k = 0; k < CL_MAX_RXN; ++k) {
                const XmlNode* r = rt->find("reaction" + std::to_string(k));
                if (!r) break;
                cl_rxn& x = c.rxn[c.n_rxn++];
                x.microbe = r->has("microbe") ? (int32_t)(*r)["microbe"].integer() : -1;
                x.k = (*r)["k"].num();
                x.yield = num_or(*r, {"yield"}, 0.0);
                x.ksp = num_or(*r, {"ksp"}, 0.0);
                if (r->has("monod"))
                    for (auto& pv : pairs((*r)["monod"])) {
                        if (x.n_monod == CL_MAX_MONOD) throw std::runtime_error("too many Monod terms in " + r->path);
                        x.monod_s[x.n_monod] = pv.first; x.monod_ks[x.n_monod] = pv.second; ++x.n_monod;
                    }
                if (r->has("mass"))
                    for (double v : (*r)["mass"].nums()) {
                        if (x.n_mass == 2) throw std::runtime_error("at most two mass-action terms in " + r->path);
                        x.mass_s[x.n_mass++] = (int32_t)v;
                    }
                if (r->has("nu"))
                    for (auto& pv : pairs((*r)["nu"])) {
                        if (pv.first < 0 || pv.first >= S) throw std::runtime_error("nu index out of range in " + r->path);
                        x.nu[pv.first] = pv.second;
                    }
            }
        }
        int n_bio = 0, n_abio = 0;
        for (int k = 0; k < c.n_rxn; ++k) (c.rxn[k].microbe >= 0 ? n_bio : n_abio)++;
        c.enable_kinetics = enable_kinetics && M > 0 ? 1 : 0;
        c.enable_abiotic = enable_abiotic ? 1 : 0;
        if (enable_kinetics && M > 0 && n_bio == 0)
            run.notes.push_back("kinetics enabled but <rate_table> has no biotic reaction: only biomass decay runs");
        if (enable_abiotic && n_abio == 0)
            run.notes.push_back("abiotic kinetics enabled but <rate_table> has no abiotic reaction");

        // equilibrium (complab_functions.hh:1245-1320)
        if (const XmlNode* eq = opt(P, {"equilibrium"}); eq && eq->has("enabled") && (*eq)["enabled"].flag()) {
            c.use_equilibrium = 1;
            cl_eq_system& e = c.eq;
            const std::vector<std::string> comps = eq->has("components") ? (*eq)["components"].words()
                                                                          : std::vector<std::string>{};
            if (comps.empty() || (int)comps.size() > CL_MAX_COMP) throw std::runtime_error("equilibrium needs 1.." + std::to_string(CL_MAX_COMP) + " components");
            e.n_comp = (int32_t)comps.size();
            e.n_species = S;
            for (int j = 0; j < e.n_comp; ++j) {
                e.comp_species[j] = -1;
                for (int s = 0; s < S; ++s) if (run.subs_names[s] == comps[j]) { e.comp_species[j] = s; break; }
            }
            for (int s = 0; s < S; ++s) {
                const std::string tag = "species" + std::to_string(s);
                if (const XmlNode* row = opt(*eq, {"stoichiometry", tag.c_str()})) {
                    const std::vector<double> v = row->nums();
                    if ((int)v.size() == e.n_comp) for (int j = 0; j < e.n_comp; ++j) e.stoich[s][j] = v[j];
                    else run.notes.push_back(tag + " stoichiometry length differs from the component count: zeros");
                }
                if (const XmlNode* lk = opt(*eq, {"logK", tag.c_str()})) e.logk[s] = lk->num();
            }
            e.max_iter = 200;               // EquilibriumChemistry's limit (complab.cpp:424)
            e.tol = 1e-10;
            e.warm_iter = 8;
            // extension: <warm_start>previous</warm_start> starts each voxel's
            // Newton from its last converged solution (reference: cold start)
            if (const XmlNode* w = eq->find("warm_start"))
                c.eq_warm_previous = lower(w->str()) == "previous" ? 1 : 0;
            // extension: <solver>pcf</solver> runs the reference's live solver
            // (PCF + Anderson, depth 4: complab.cpp:423-425) instead of Newton
            if (const XmlNode* sv = eq->find("solver")) {
                const std::string v = lower(sv->str());
                if (v == "pcf") e.solver = CL_EQ_SOLVER_PCF;
                else if (v == "newton") e.solver = CL_EQ_SOLVER_NEWTON;
                else throw std::runtime_error("equilibrium solver must be newton or pcf");
            }
            e.anderson_depth = 4;
        }

        // precipitation (complab.cpp:272-294)
        if (const XmlNode* pr = opt(P, {"precipitation"}); pr && pr->has("enabled") && (*pr)["enabled"].flag()) {
            c.precip_enabled = 1;
            c.precip_substrate = (int32_t)num_or(*pr, {"solid_substrate"}, -1);
            c.max_precip_rho = num_or(*pr, {"max_precipRho"}, 1e30);
            c.abiotic_surface_only = (int32_t)num_or(*pr, {"surface_only"}, 1);
            c.precip_code = c.solid_code;
            run.precip_interval = (long)num_or(*pr, {"update_interval"}, 200);
            if (num_or(*pr, {"perm_ratio"}, 0.0) > kThrd)
                run.notes.push_back("precipitation perm_ratio > 0: sealed voxels stay NoDynamics for the flow here");
        }

        // dissolution (complab.cpp:297-375)
        if (const XmlNode* di = opt(P, {"dissolution"}); di && di->has("enabled") && (*di)["enabled"].flag()) {
            c.dissol_enabled = 1;
            c.reopen_fraction = num_or(*di, {"reopen_fraction"}, 0.9);
            c.dissol_surface_only = (int32_t)num_or(*di, {"surface_only"}, 1);
            c.dissol_apply_at_walls = (int32_t)num_or(*di, {"apply_at_walls"}, 0);
            run.dissol_interval = (long)num_or(*di, {"update_interval"}, 200);
            for (int k = 0; k < CL_MAX_PHASES; ++k) {
                const XmlNode* ph = di->find("phase" + std::to_string(k));
                if (!ph || !ph->has("material_number")) break;
                cl_phase& q = c.phases[c.n_phases];
                q.id = c.n_phases + 1;
                q.material = (int32_t)(*ph)["material_number"].integer();
                q.substrate = (int32_t)num_or(*ph, {"substrate"}, -1);
                q.full_density = num_or(*ph, {"full_density"}, 0.0);
                q.initial_fill = num_or(*ph, {"initial_fill"}, 0.0);
                q.is_precipitate = ph->has("is_precipitate") && (*ph)["is_precipitate"].flag() ? 1 : 0;
                const XmlNode* rsrc = ph;
                if (!ph->has("rate_k") && RP)
                    if (const XmlNode* rd = RP->find("dissolution"))
                        if (const XmlNode* rp = rd->find("phase" + std::to_string(k))) rsrc = rp;
                q.k = num_or(*rsrc, {"rate_k"}, 0.0);
                if (rsrc->has("rate_mass"))
                    for (double v : (*rsrc)["rate_mass"].nums()) if (q.n_mass < 2) q.mass_s[q.n_mass++] = (int32_t)v;
                if (rsrc->has("rate_nu"))
                    for (auto& pv : pairs((*rsrc)["rate_nu"])) if (pv.first >= 0 && pv.first < S) q.nu[pv.first] = pv.second;
                if (q.is_precipitate) c.precip_phase_id = q.id;
                ++c.n_phases;
            }
            if (c.n_phases == 0) throw std::runtime_error("<dissolution> is enabled but no <phase0> block was given");
        }
        // cellular automaton (complab_functions.hh:1167-1186): every sessile
        // microbe is CA- or finite-difference-solved; both keep the mask and
        // total-biomass state of the CA (finite differences run its mask
        // update around their diffusion step, complab.cpp:1716-1731); a
        // microbe's material code is the first of its material numbers
        // (bio_dynamics[m][0])
        int n_ca = 0, n_fd = 0;
        for (int m = 0; m < M; ++m) { n_ca += run.carried[m] ? 0 : 1; n_fd += run.fd[m]; }
        if (n_fd > 0 && n_fd != n_ca)
            throw std::runtime_error("finite-difference and cellular-automaton microbes in one run are not supported");
        if (n_ca > 0) {
            const XmlNode& mic = P["microbiology"];
            if (!mic.has("thrd_biofilm_fraction"))
                throw std::runtime_error("thrd_biofilm_fraction must be defined when solver_type is Cellular Automata");
            c.ca_thrd_frac = mic["thrd_biofilm_fraction"].num();
            if (mic.has("maximum_biomass_density")) c.ca_bmax = mic["maximum_biomass_density"].num();
            else if (M == 1)
                throw std::runtime_error("maximum_biomass_density must be defined when solver_type is Cellular Automata");
            else c.ca_bmax = 999999999.;
            c.ca_half = 0;
            if (mic.has("CA_method")) {
                const std::string h = lower(mic["CA_method"].str());
                if (h == "fraction" || h == "0" || h == "no") c.ca_half = 0;
                else if (h == "half" || h == "1" || h == "yes") c.ca_half = 1;
                else throw std::runtime_error("CA_method (" + h + ") should be either half or fraction");
            }
            for (int m = 0; m < M; ++m) {
                if (run.carried[m]) continue;            // the CA moves sessile biomass only
                if (run.bio_materials[m].empty())
                    throw std::runtime_error("microbe" + std::to_string(m) + " has no material number for its biofilm");
                c.microbe_code[m] = run.bio_materials[m][0];
            }
            // std::srand(time) in the reference; a fixed seed of the counter-based generator here
            c.ca_seed = mic.has("ca_seed") ? (uint64_t)mic["ca_seed"].integer() : 1;
            c.ca_enabled = 1;
        }
        return 0;
    } catch (const std::exception& e) {
        err = e.what();
        return -1;
    }
}


// nu of the finite-difference step over refNu: bioNUinPore[0] / refNu =
// D_bmass_pore[0] / D_pore[0] where microbe 0's coefficient is positive, else 0
// (complab.cpp:731-736)
double fd_nu_ratio(const HostRun& r) {
    return (r.D_bmass_pore0 > 0 && !r.D_pore.empty() && r.D_pore[0] > 0) ? r.D_bmass_pore0 / r.D_pore[0] : 0.0;
}

std::string run_json(const HostRun& r) {
    const cl_config& c = r.cfg;
    std::ostringstream o;
    o.precision(17);
    auto arr = [&](const double* v, int n) {
        o << "[";
        for (int i = 0; i < n; ++i) o << (i ? ", " : "") << v[i];
        o << "]";
    };
    auto iarr = [&](const int32_t* v, int n) {
        o << "[";
        for (int i = 0; i < n; ++i) o << (i ? ", " : "") << v[i];
        o << "]";
    };
    o << "{\"nx\": " << c.nx << ", \"ny\": " << c.ny << ", \"nz\": " << c.nz
      << ", \"dx\": " << r.dx << ", \"geometry\": \"" << r.geom_file << "\""
      << ", \"solid\": " << c.solid_code << ", \"bounce_back\": " << c.bb_code << ", \"pore\": ";
    iarr(c.pore_codes, c.n_pore_codes);
    o << ", \"bio\": ";
    iarr(c.bio_codes, c.n_bio_codes);
    o << ", \"tau\": " << r.tau << ", \"delta_P\": " << r.delta_P << ", \"Pe\": " << r.Pe
      << ", \"charcs_length\": " << r.charcs_length << ", \"rho_out\": " << c.rho_out
      << ", \"ns_max_iT1\": " << r.ns_max1 << ", \"ns_converge_iT1\": " << r.ns_conv1
      << ", \"ade_max_iT\": " << r.ade_max << ", \"ns_update_interval\": " << r.ns_update_interval
      << ", \"ade_update_interval\": " << r.ade_update_interval << ", \"ns_max_iT2\": " << r.ns_max2
      << ", \"ns_converge_iT2\": " << r.ns_conv2 << ", \"precip_interval\": " << r.precip_interval
      << ", \"dissol_interval\": " << r.dissol_interval << ", \"vtk_interval\": " << r.vtk_interval << ", \"chk_interval\": " << r.chk_interval
      << ", \"n_solutes\": " << c.n_solutes << ", \"names\": [";
    for (size_t i = 0; i < r.subs_names.size(); ++i) o << (i ? ", " : "") << "\"" << r.subs_names[i] << "\"";
    o << "], \"c0\": ";
    arr(c.c0, c.n_solutes);
    o << ", \"immobile\": ";
    iarr(c.immobile, c.n_solutes);
    o << ", \"left_type\": ";
    iarr(c.left_type, c.n_solutes);
    o << ", \"left_value\": ";
    arr(c.left_value, c.n_solutes);
    o << ", \"right_type\": ";
    iarr(c.right_type, c.n_solutes);
    o << ", \"right_value\": ";
    arr(c.right_value, c.n_solutes);
    o << ", \"omega_pore\": ";
    arr(c.omega_pore, c.n_solutes);
    o << ", \"omega_bio\": ";
    arr(c.omega_bio, c.n_solutes);
    o << ", \"dt\": " << c.dt << ", \"n_microbes\": " << c.n_microbes
      << ", \"enable_kinetics\": " << c.enable_kinetics << ", \"enable_abiotic\": " << c.enable_abiotic
      << ", \"n_rxn\": " << c.n_rxn << ", \"use_equilibrium\": " << c.use_equilibrium
      << ", \"n_comp\": " << c.eq.n_comp << ", \"eq_solver\": \"" << (c.eq.solver == CL_EQ_SOLVER_PCF ? "pcf" : "newton")
      << "\", \"comp_species\": ";
    iarr(c.eq.comp_species, c.eq.n_comp);
    o << ", \"logk\": ";
    arr(c.eq.logk, c.use_equilibrium ? c.n_solutes : 0);
    o << ", \"precip_enabled\": " << c.precip_enabled << ", \"precip_substrate\": " << c.precip_substrate
      << ", \"max_precip_rho\": " << c.max_precip_rho << ", \"dissol_enabled\": " << c.dissol_enabled
      << ", \"n_phases\": " << c.n_phases << ", \"precip_phase_id\": " << c.precip_phase_id
      << ", \"ca_enabled\": " << c.ca_enabled << ", \"ca_half\": " << c.ca_half
      << ", \"ca_bmax\": " << c.ca_bmax << ", \"ca_thrd_frac\": " << c.ca_thrd_frac
      << ", \"ca_seed\": " << c.ca_seed << ", \"microbe_code\": ";
    iarr(c.microbe_code, c.n_microbes);
    // per microbe: its biofilm materials and the initial density on each
    o << ", \"bio_materials\": [";
    for (size_t m = 0; m < r.bio_materials.size(); ++m) {
        o << (m ? ", " : "") << "[";
        for (size_t k = 0; k < r.bio_materials[m].size(); ++k) o << (k ? ", " : "") << r.bio_materials[m][k];
        o << "]";
    }
    // finite-difference microbes, and nu / refNu of their step (bioNUinPore[0])
    o << "], \"fd\": [";
    for (size_t m = 0; m < r.fd.size(); ++m) o << (m ? ", " : "") << r.fd[m];
    o << "], \"fd_nu_ratio\": " << fd_nu_ratio(r) << ", \"n_srg\": " << c.n_srg << ", \"surrogate_files\": [";
    for (size_t k = 0; k < r.srg_files.size(); ++k) o << (k ? ", " : "") << "\"" << r.srg_files[k] << "\"";
    o << "]";
    o << ", \"microbe_names\": [";
    for (size_t m = 0; m < r.microbe_names.size(); ++m) o << (m ? ", " : "") << "\"" << r.microbe_names[m] << "\"";
    o << "], \"b0\": [";
    for (size_t m = 0; m < r.b0.size(); ++m) {
        o << (m ? ", " : "") << "[";
        for (size_t k = 0; k < r.b0[m].size(); ++k) o << (k ? ", " : "") << r.b0[m][k];
        o << "]";
    }
    o << "], \"notes\": [";
    for (size_t i = 0; i < r.notes.size(); ++i) o << (i ? ", " : "") << "\"" << r.notes[i] << "\"";
    o << "]}";
    return o.str();
}

}  // namespace clhost
