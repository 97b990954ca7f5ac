// complab_io.h -- the host driver's output formats: VTK ImageData files in
// the reference's naming, and a documented checkpoint the driver restarts from.
//
// VTI (writeAdvVTI / writeNsVTI, src/complab_functions.hh:86-125): one
// VTK XML ImageData file per field and output step over the interior planes
// x = 1..nx-2 (the reference's Box3D(1, nx-2, 0, ny-1, 0, nz-1)), spacing 1,
// named <name>_<step, 7 digits>.vti: "Density" (FP64) for every solute, every
// microbe and the material numbers, "velocityNorm" and "velocity" (FP32) in
// nsLattice_<step>.vti.  Point data is x fastest, as VTK orders it; inline
// binary, base64 with a UInt64 byte-count header.
//
// Checkpoint (the reference saves Palabos binary blocks, complab.cpp:1237-1247,
// a format of Palabos's own): a folder chk_<steps>/ with checkpoint.json (the
// sizes, the steps done, the calibrated pressure, dt and relaxation of the
// run) and raw little-endian arrays in site order n = (x*ny + y)*nz + z:
//   mask.u8              material numbers (N bytes)
//   dynamics.u8          2*N dynamics classes, the flow's then the solutes'
//                        (they follow the node conversions' dynamics switches)
//   flow.f32             19*N flow deviations f_i - t_i, natural order (when a flow exists)
//   solute_<s>.f32       7*N populations of a mobile solute, natural order
//   solute_<s>.f64       N inventory values of an immobile solute
//   biomass_<m>.f64      N sessile biomass values
//   phase.f64            N phase ids (with dissolution)
//   eq_start.f64         2*n_comp*N Newton warm starts (with eq_warm_previous)
// Restarting from it reproduces the uninterrupted run bit for bit (the
// cellular automaton's age field is not saved: a CA run restarts with its
// ages recomputed from the mask).
#pragma once
#include <string>
#include <vector>

#include "../../include/complab_gpu.h"
#include "complab_xml.h"

namespace clhost {

struct VtiArray {
    std::string name;
    int comps;                       // 1 or 3
    bool f64;                        // Float64 (else Float32)
    std::vector<double> data;        // comps arrays of N values each, site order
};

// Writes one ImageData file; returns false with a message in err.
bool write_vti(const std::string& path, int nx, int ny, int nz, const std::vector<VtiArray>& arrays,
               std::string& err);

// The reference's file name: <name><step, zero-padded to 7 digits>.vti
std::string vti_name(const std::string& prefix, long step);

struct Checkpoint {
    long steps = 0;                  // transport steps done when it was written
    double rho_in = 1.0, rho_out = 1.0, dt = 1.0, delta_P = 0.0;
    std::vector<double> omega_pore, omega_bio;
    bool has_flow = false;
};

bool save_checkpoint(cl_ctx* h, const HostRun& run, const Checkpoint& chk, const std::string& dir, std::string& err);
// header and geometry (before the context exists)
bool read_checkpoint(const std::string& dir, const HostRun& run, Checkpoint& chk, std::vector<uint8_t>& mask,
                     std::string& err);
// the dynamics classes (right after the mask upload)
bool restore_dynamics(cl_ctx* h, const HostRun& run, const std::string& dir, std::string& err);
// the flow populations (after the mask upload)
bool restore_flow(cl_ctx* h, const HostRun& run, const std::string& dir, std::string& err);
// the transport state (after cl_ade_init)
bool restore_transport(cl_ctx* h, const HostRun& run, const std::string& dir, std::string& err);

}  // namespace clhost
