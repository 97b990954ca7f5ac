// complab_io.cpp -- VTI output and checkpoints of the host driver (see complab_io.h).
#include "complab_io.h"

#include <sys/stat.h>

#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

namespace clhost {

namespace {

const char kB64[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";

void base64(const unsigned char* p, size_t n, std::string& out) {
    out.reserve(out.size() + (n + 2) / 3 * 4);
    size_t i = 0;
    for (; i + 2 < n; i += 3) {
        const unsigned v = (unsigned)p[i] << 16 | (unsigned)p[i + 1] << 8 | p[i + 2];
        out += kB64[v >> 18 & 63]; out += kB64[v >> 12 & 63]; out += kB64[v >> 6 & 63]; out += kB64[v & 63];
    }
    if (i < n) {
        unsigned v = (unsigned)p[i] << 16;
        if (i + 1 < n) v |= (unsigned)p[i + 1] << 8;
        out += kB64[v >> 18 & 63];
        out += kB64[v >> 12 & 63];
        out += i + 1 < n ? kB64[v >> 6 & 63] : '=';
        out += '=';
    }
}

bool write_raw(const std::string& path, const void* p, size_t bytes, std::string& err) {
    std::ofstream o(path, std::ios::binary);
    o.write(static_cast<const char*>(p), (std::streamsize)bytes);
    if (!o) { err = "cannot write " + path; return false; }
    return true;
}

bool read_raw(const std::string& path, void* p, size_t bytes, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    f.read(static_cast<char*>(p), (std::streamsize)bytes);
    if (f.gcount() != (std::streamsize)bytes) { err = path + " is shorter than " + std::to_string(bytes) + " bytes"; return false; }
    return true;
}

bool ok(int st, const char* what, std::string& err) {
    if (st >= 0) return true;
    err = std::string(what) + " failed: " + cl_last_error();
    return false;
}

// the numbers after "key": in a flat JSON object written by save_checkpoint
std::vector<double> json_nums(const std::string& js, const std::string& key) {
    std::vector<double> v;
    const size_t k = js.find("\"" + key + "\":");
    if (k == std::string::npos) return v;
    size_t p = k + key.size() + 3;
    while (p < js.size() && std::isspace((unsigned char)js[p])) ++p;
    const bool arr = p < js.size() && js[p] == '[';
    if (arr) ++p;
    while (p < js.size()) {
        char* end = nullptr;
        const double d = std::strtod(js.c_str() + p, &end);
        if (end == js.c_str() + p) break;
        v.push_back(d);
        p = (size_t)(end - js.c_str());
        while (p < js.size() && (std::isspace((unsigned char)js[p]) || js[p] == ',')) ++p;
        if (!arr || (p < js.size() && js[p] == ']')) break;
    }
    return v;
}

}  // namespace

std::string vti_name(const std::string& prefix, long step) {
    char num[32];
    std::snprintf(num, sizeof num, "%07ld", step);
    return prefix + num + ".vti";
}

bool write_vti(const std::string& path, int nx, int ny, int nz, const std::vector<VtiArray>& arrays,
               std::string& err) {
    const int mx = nx - 2;
    const size_t N = (size_t)nx * ny * nz, M = (size_t)mx * ny * nz;
    std::ofstream o(path, std::ios::binary);
    if (!o) { err = "cannot write " + path; return false; }
    o << "<?xml version=\"1.0\"?>\n"
      << "<VTKFile type=\"ImageData\" version=\"1.0\" byte_order=\"LittleEndian\" header_type=\"UInt64\">\n"
      << "  <ImageData WholeExtent=\"0 " << mx - 1 << " 0 " << ny - 1 << " 0 " << nz - 1
      << "\" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n"
      << "    <Piece Extent=\"0 " << mx - 1 << " 0 " << ny - 1 << " 0 " << nz - 1 << "\">\n"
      << "      <PointData>\n";
    for (const VtiArray& a : arrays) {
        if (a.data.size() != (size_t)a.comps * N) { err = "array " + a.name + " has the wrong size"; return false; }
        const size_t esz = a.f64 ? 8 : 4;
        std::vector<unsigned char> buf(8 + M * a.comps * esz);
        const uint64_t nbytes = (uint64_t)(M * a.comps * esz);
        std::memcpy(buf.data(), &nbytes, 8);
        unsigned char* q = buf.data() + 8;
        // VTK point order: x fastest, then y, then z; components interleaved
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 1; x <= mx; ++x) {
                    const size_t n = ((size_t)x * ny + y) * nz + z;
                    for (int c = 0; c < a.comps; ++c) {
                        const double v = a.data[(size_t)c * N + n];
                        if (a.f64) { std::memcpy(q, &v, 8); q += 8; }
                        else { const float f = (float)v; std::memcpy(q, &f, 4); q += 4; }
                    }
                }
        std::string enc;
        base64(buf.data(), buf.size(), enc);
        o << "        <DataArray type=\"" << (a.f64 ? "Float64" : "Float32") << "\" Name=\"" << a.name
          << "\" NumberOfComponents=\"" << a.comps << "\" format=\"binary\">\n          " << enc
          << "\n        </DataArray>\n";
    }
    o << "      </PointData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n";
    if (!o) { err = "cannot write " + path; return false; }
    return true;
}

bool save_checkpoint(cl_ctx* h, const HostRun& run, const Checkpoint& chk, const std::string& dir, std::string& err) {
    const cl_config& c = run.cfg;
    const size_t N = (size_t)c.nx * c.ny * c.nz;
    mkdir(dir.c_str(), 0777);
    std::vector<uint8_t> mask(N);
    if (!ok(cl_download_mask(h, mask.data()), "cl_download_mask", err)) return false;
    if (!write_raw(dir + "/mask.u8", mask.data(), N, err)) return false;
    {
        std::vector<double> cd(N);
        std::vector<uint8_t> cls(2 * N);
        for (int k = 0; k < 2; ++k) {
            if (!ok(cl_get_field(h, CL_FIELD_DYNAMICS, k, cd.data()), "cl_get_field", err)) return false;
            for (size_t n = 0; n < N; ++n) cls[k * N + n] = (uint8_t)cd[n];
        }
        if (!write_raw(dir + "/dynamics.u8", cls.data(), 2 * N, err)) return false;
    }
    if (chk.has_flow) {
        std::vector<float> f(19 * N);
        if (!ok(cl_get_flow_populations(h, f.data()), "cl_get_flow_populations", err)) return false;
        if (!write_raw(dir + "/flow.f32", f.data(), f.size() * 4, err)) return false;
    }
    std::vector<float> g(7 * N);
    std::vector<double> d(N);
    for (int s = 0; s < c.n_solutes; ++s) {
        if (!c.immobile[s]) {
            if (!ok(cl_get_solute_populations(h, s, g.data()), "cl_get_solute_populations", err)) return false;
            if (!write_raw(dir + "/solute_" + std::to_string(s) + ".f32", g.data(), g.size() * 4, err)) return false;
        } else {
            if (!ok(cl_get_field(h, CL_FIELD_CONC, s, d.data()), "cl_get_field", err)) return false;
            if (!write_raw(dir + "/solute_" + std::to_string(s) + ".f64", d.data(), N * 8, err)) return false;
        }
    }
    for (int m = 0; m < c.n_microbes; ++m) {
        if (!ok(cl_get_field(h, CL_FIELD_BIOMASS, m, d.data()), "cl_get_field", err)) return false;
        if (!write_raw(dir + "/biomass_" + std::to_string(m) + ".f64", d.data(), N * 8, err)) return false;
    }
    if (c.dissol_enabled) {
        if (!ok(cl_get_field(h, CL_FIELD_PHASE, 0, d.data()), "cl_get_field", err)) return false;
        if (!write_raw(dir + "/phase.f64", d.data(), N * 8, err)) return false;
    }
    const int nc = c.use_equilibrium && c.eq_warm_previous ? c.eq.n_comp : 0;
    if (nc > 0) {
        std::ofstream o(dir + "/eq_start.f64", std::ios::binary);
        for (int j = 0; j < 2 * nc; ++j) {
            if (!ok(cl_get_field(h, CL_FIELD_EQ_START, j, d.data()), "cl_get_field", err)) return false;
            o.write(reinterpret_cast<const char*>(d.data()), (std::streamsize)(N * 8));
        }
        if (!o) { err = "cannot write " + dir + "/eq_start.f64"; return false; }
    }
    std::ofstream js(dir + "/checkpoint.json");
    js.precision(17);
    js << "{\"format\": \"complab-b200 checkpoint\", \"version\": 1, \"nx\": " << c.nx << ", \"ny\": " << c.ny
       << ", \"nz\": " << c.nz << ", \"steps\": " << chk.steps << ", \"n_solutes\": " << c.n_solutes
       << ", \"n_microbes\": " << c.n_microbes << ", \"n_comp_warm\": " << nc << ", \"has_flow\": "
       << (chk.has_flow ? 1 : 0) << ", \"rho_in\": " << chk.rho_in << ", \"rho_out\": " << chk.rho_out
       << ", \"delta_P\": " << chk.delta_P << ", \"dt\": " << chk.dt << ", \"omega_pore\": [";
    for (size_t s = 0; s < chk.omega_pore.size(); ++s) js << (s ? ", " : "") << chk.omega_pore[s];
    js << "], \"omega_bio\": [";
    for (size_t s = 0; s < chk.omega_bio.size(); ++s) js << (s ? ", " : "") << chk.omega_bio[s];
    js << "]}\n";
    if (!js) { err = "cannot write " + dir + "/checkpoint.json"; return false; }
    return true;
}

bool read_checkpoint(const std::string& dir, const HostRun& run, Checkpoint& chk, std::vector<uint8_t>& mask,
                     std::string& err) {
    std::ifstream f(dir + "/checkpoint.json");
    if (!f) { err = "no checkpoint.json in " + dir; return false; }
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string js = ss.str();
    if (js.find("complab-b200 checkpoint") == std::string::npos) { err = dir + " is not a checkpoint"; return false; }
    const cl_config& c = run.cfg;
    auto one = [&](const char* k, double& v) {
        const std::vector<double> a = json_nums(js, k);
        if (a.size() != 1) return false;
        v = a[0];
        return true;
    };
    double nx = 0, ny = 0, nz = 0, S = 0, M = 0, steps = 0, hf = 0;
    if (!one("nx", nx) || !one("ny", ny) || !one("nz", nz) || !one("n_solutes", S) || !one("n_microbes", M) ||
        !one("steps", steps) || !one("has_flow", hf) || !one("rho_in", chk.rho_in) || !one("rho_out", chk.rho_out) ||
        !one("dt", chk.dt) || !one("delta_P", chk.delta_P)) {
        err = "checkpoint.json in " + dir + " lacks a field";
        return false;
    }
    if ((int)nx != c.nx || (int)ny != c.ny || (int)nz != c.nz || (int)S != c.n_solutes || (int)M != c.n_microbes) {
        err = "the checkpoint in " + dir + " does not match CompLaB.xml's sizes";
        return false;
    }
    chk.steps = (long)steps;
    chk.has_flow = hf != 0;
    chk.omega_pore = json_nums(js, "omega_pore");
    chk.omega_bio = json_nums(js, "omega_bio");
    if ((int)chk.omega_pore.size() != c.n_solutes || (int)chk.omega_bio.size() != c.n_solutes) {
        err = "checkpoint.json in " + dir + " has the wrong number of relaxation frequencies";
        return false;
    }
    mask.assign((size_t)c.nx * c.ny * c.nz, 0);
    return read_raw(dir + "/mask.u8", mask.data(), mask.size(), err);
}

bool restore_dynamics(cl_ctx* h, const HostRun& run, const std::string& dir, std::string& err) {
    const cl_config& c = run.cfg;
    const size_t N = (size_t)c.nx * c.ny * c.nz;
    std::vector<uint8_t> cls(2 * N);
    if (!read_raw(dir + "/dynamics.u8", cls.data(), cls.size(), err)) return false;
    std::vector<double> cd(N);
    for (int k = 0; k < 2; ++k) {
        for (size_t n = 0; n < N; ++n) cd[n] = cls[k * N + n];
        if (!ok(cl_set_field(h, CL_FIELD_DYNAMICS, k, cd.data()), "cl_set_field", err)) return false;
    }
    return true;
}

bool restore_flow(cl_ctx* h, const HostRun& run, const std::string& dir, std::string& err) {
    const cl_config& c = run.cfg;
    std::vector<float> f((size_t)19 * c.nx * c.ny * c.nz);
    if (!read_raw(dir + "/flow.f32", f.data(), f.size() * 4, err)) return false;
    return ok(cl_set_flow_populations(h, f.data()), "cl_set_flow_populations", err);
}

bool restore_transport(cl_ctx* h, const HostRun& run, const std::string& dir, std::string& err) {
    const cl_config& c = run.cfg;
    const size_t N = (size_t)c.nx * c.ny * c.nz;
    std::vector<float> g(7 * N);
    std::vector<double> d(N);
    for (int s = 0; s < c.n_solutes; ++s) {
        const std::string base = dir + "/solute_" + std::to_string(s);
        if (!c.immobile[s]) {
            if (!read_raw(base + ".f32", g.data(), g.size() * 4, err)) return false;
            if (!ok(cl_set_solute_populations(h, s, g.data()), "cl_set_solute_populations", err)) return false;
        } else {
            if (!read_raw(base + ".f64", d.data(), N * 8, err)) return false;
            if (!ok(cl_set_field(h, CL_FIELD_CONC, s, d.data()), "cl_set_field", err)) return false;
        }
    }
    for (int m = 0; m < c.n_microbes; ++m) {
        if (!read_raw(dir + "/biomass_" + std::to_string(m) + ".f64", d.data(), N * 8, err)) return false;
        if (!ok(cl_set_field(h, CL_FIELD_BIOMASS, m, d.data()), "cl_set_field", err)) return false;
    }
    if (c.dissol_enabled) {
        if (!read_raw(dir + "/phase.f64", d.data(), N * 8, err)) return false;
        if (!ok(cl_set_field(h, CL_FIELD_PHASE, 0, d.data()), "cl_set_field", err)) return false;
    }
    const int nc = c.use_equilibrium && c.eq_warm_previous ? c.eq.n_comp : 0;
    if (nc > 0) {
        std::ifstream f(dir + "/eq_start.f64", std::ios::binary);
        if (!f) { err = "cannot open " + dir + "/eq_start.f64"; return false; }
        for (int j = 0; j < 2 * nc; ++j) {
            f.read(reinterpret_cast<char*>(d.data()), (std::streamsize)(N * 8));
            if (f.gcount() != (std::streamsize)(N * 8)) { err = dir + "/eq_start.f64 is short"; return false; }
            if (!ok(cl_set_field(h, CL_FIELD_EQ_START, j, d.data()), "cl_set_field", err)) return false;
        }
    }
    return true;
}

}  // namespace clhost
