// complab_xml.h -- CompLaB.xml -> cl_config for the host driver.
//
// Reads the schema of the reference's initialize_complab
// (src/complab_functions.hh:621-1349) and of the blocks complab.cpp parses
// itself (<immobile>, <precipitation>, <dissolution>; complab.cpp:244-375),
// with the same defaults, for the parts of the hot path this library runs.
// Two blocks extend the schema where the reference compiles C++ instead of
// reading XML: <rate_table> stands for defineKinetics.hh /
// defineAbioticKinetics.hh (the table form of cl_rxn), and <rate_k>,
// <rate_mass>, <rate_nu> inside a dissolution <phaseN> stand for
// defineDissolutionRate.  Because the reference keeps those laws in compiled
// headers, its own example inputs carry none of them: a second file given as
// `rates` (root <parameters>, holding <rate_table> and/or
// <dissolution><phaseN><rate_k>...) supplies the blocks the main file lacks.
#pragma once
#include <string>
#include <vector>
#include "../../include/complab_gpu.h"

namespace clhost {

struct HostRun {
    cl_config cfg{};
    std::string xml_dir, input_dir, output_dir, geom_file;
    // LB_numerics
    double dx = 0.0;                 // m, after the <unit> scaling
    double delta_P = 0.0, Pe = 0.0, tau = 0.8, charcs_length = 0.0;   // charcs_length in lattice units
    long ns_max1 = 100000, ns_max2 = 100000, ade_max = 10000000;
    long ns_update_interval = 1, ade_update_interval = 1;   // geometry-change dynamics / flow updates
    double ns_conv1 = 1e-8, ns_conv2 = 1e-6;
    long vtk_interval = 0, chk_interval = 0;     // <IO> save_VTK_interval, save_CHK_interval
    std::string mask_filename = "maskLattice";
    // chemistry / microbiology
    std::vector<std::string> subs_names, microbe_names;
    std::vector<double> D_pore, D_bfilm;
    std::vector<double> D_bfilm_ref;                 // divisor of the biofilm relaxation (complab.cpp:725, :738)
    std::vector<int> carried;                        // per microbe: 1 if solved by LBM (a carrier solute)
    std::vector<int> fd;                             // per microbe: 1 if solved by finite differences (sessile)
    bool enable_surrogate = false;                   // <enable_surrogate>
    std::vector<std::string> srg_files;              // network of each surrogate organism, in order (--surrogate)
    double D_bmass_pore0 = -99.0;                    // microbe 0's biomass pore diffusion (bioNUinPore[0], complab.cpp:731-736)
    std::vector<std::vector<int>> bio_materials;    // per microbe: its biofilm material numbers
    std::vector<std::vector<double>> b0;            // per microbe: initial density per material
    bool biotic_mode = true;
    // geometry updates
    long precip_interval = 1, dissol_interval = 200;
    std::vector<std::string> notes;                  // what the driver does not run, said once
};

// Returns 0 on success; on failure -1 with a message in err.
int read_complab_xml(const std::string& path, HostRun& run, std::string& err, const std::string& rates = "");

// The parsed run as JSON (used by --print-config and the tests).
// nu of the finite-difference biomass step over refNu (bioNUinPore[0] / refNu)
double fd_nu_ratio(const HostRun& r);
std::string run_json(const HostRun& run);

}  // namespace clhost
