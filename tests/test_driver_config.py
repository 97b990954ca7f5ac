"""The host driver's CompLaB.xml reader (CPU): the schema, defaults and unit
handling of the reference's initialize_complab, checked through
`complab_b200 --print-config` on XML files written here."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "complb3d-lattice-boltzmann-fba-surrogate-cobrapy-glpk_b200", "complab_b200")

CASE = """<?xml version="1.0" ?>
<!-- a small abiotic case: A -> P on wall-adjacent voxels, P immobile -->
<parameters>
    <path><input_path>input</input_path><output_path>output</output_path></path>
    <simulation_mode>
        <biotic_mode>false</biotic_mode>
        <enable_abiotic_kinetics>true</enable_abiotic_kinetics>
    </simulation_mode>
    <LB_numerics>
        <domain>
            <nx>{nx}</nx><ny>{ny}</ny><nz>{nz}</nz>
            <dx>10</dx><unit>um</unit>
            <characteristic_length>{L}</characteristic_length>
            <filename>geometry.dat</filename>
            <material_numbers><pore>2</pore><solid>0</solid><bounce_back>1</bounce_back></material_numbers>
        </domain>
        <delta_P>{dP}</delta_P>
        <Peclet>{Pe}</Peclet>
        <tau>0.8</tau>
        <iteration>
            <ns_max_iT1>3000</ns_max_iT1>
            <ns_converge_iT1>1e-7</ns_converge_iT1>
            <ade_max_iT>{steps}</ade_max_iT>
        </iteration>
    </LB_numerics>
    <chemistry>
        <number_of_substrates>2</number_of_substrates>
        <substrate0>
            <name_of_substrates>A</name_of_substrates>
            <initial_concentration>0.1</initial_concentration>
            <substrate_diffusion_coefficients><in_pore>1e-9</in_pore><in_biofilm>5e-10</in_biofilm></substrate_diffusion_coefficients>
            <left_boundary_type>Dirichlet</left_boundary_type><left_boundary_condition>1.0</left_boundary_condition>
            <right_boundary_type>Neumann</right_boundary_type><right_boundary_condition>0</right_boundary_condition>
        </substrate0>
        <substrate1>
            <name_of_substrates>P</name_of_substrates>
            <immobile>true</immobile>
            <left_boundary_type>Neumann</left_boundary_type><left_boundary_condition>0</left_boundary_condition>
            <right_boundary_type>Neumann</right_boundary_type><right_boundary_condition>0</right_boundary_condition>
        </substrate1>
    </chemistry>
    <rate_table>
        <reaction0><k>0.05</k><mass>0</mass><nu>0:-1 1:1</nu></reaction0>
    </rate_table>
    <precipitation>
        <enabled>true</enabled><solid_substrate>1</solid_substrate><max_precipRho>0.02</max_precipRho>
        <surface_only>1</surface_only><update_interval>5</update_interval>
    </precipitation>
</parameters>
"""


def write_case(tmp, nx=10, ny=8, nz=8, Pe=0.0, dP=0.0, L=8, steps=20, mask=None):
    import numpy as np
    os.makedirs(os.path.join(tmp, "input"), exist_ok=True)
    xml = os.path.join(tmp, "CompLaB.xml")
    open(xml, "w").write(CASE.format(nx=nx, ny=ny, nz=nz, Pe=Pe, dP=dP, L=L * 10, steps=steps))
    if mask is None:
        mask = np.full((nx, ny, nz), 2, np.uint8)
        mask[:, :, 0] = 1
        mask[:, :, -1] = 1
    with open(os.path.join(tmp, "input", "geometry.dat"), "w") as f:
        for x in range(nx):
            f.write("\n".join(str(int(v)) for v in mask[x].reshape(-1)) + "\n")
    return xml


def driver_available():
    return os.path.exists(DRIVER)


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
def test_print_config_follows_the_schema(tmp_path):
    xml = write_case(str(tmp_path), Pe=0.0, dP=0.0)
    out = subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True, check=True).stdout
    c = json.loads(out)
    assert (c["nx"], c["ny"], c["nz"]) == (12, 8, 8)           # nx += 2 (complab_functions.hh:769)
    assert c["dx"] == pytest.approx(10e-6)                     # <unit>um
    assert c["charcs_length"] == pytest.approx(8.0)            # in lattice units
    assert c["pore"] == [2] and c["solid"] == 0 and c["bounce_back"] == 1
    assert c["names"] == ["A", "P"] and c["immobile"] == [0, 1]
    assert c["c0"] == [0.1, 0.0]
    assert c["left_type"] == [0, 1] and c["right_type"] == [1, 1]
    assert c["left_value"][0] == 1.0
    assert c["enable_abiotic"] == 1 and c["enable_kinetics"] == 0 and c["n_rxn"] == 1
    assert c["precip_enabled"] == 1 and c["precip_substrate"] == 1 and c["max_precip_rho"] == 0.02
    assert c["Pe"] == 0.0                                      # delta_P < thrd forces Pe = 0
    # without flow the transport relaxation comes from tau, dt = nu dx^2 / D0
    nu = 0.25 * (0.8 - 0.5)
    assert c["omega_pore"][0] == pytest.approx(1.0 / 0.8)
    assert c["dt"] == pytest.approx(nu * (10e-6) ** 2 / 1e-9)


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
def test_defaults_and_errors(tmp_path):
    xml = write_case(str(tmp_path), Pe=2.0, dP=1e-5)
    c = json.loads(subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True, check=True).stdout)
    assert c["Pe"] == 2.0 and c["rho_out"] == pytest.approx(1.0 - 3e-5)
    assert c["ns_max_iT1"] == 3000 and c["ns_converge_iT1"] == 1e-7
    # a required element missing: the reference terminates, the driver exits 1 with the path
    text = open(xml).read().replace("<ny>8</ny>", "")
    open(xml, "w").write(text)
    r = subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1 and "ny" in r.stderr
    r = subprocess.run([DRIVER, str(tmp_path / "absent.xml"), "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1


CA_CASE = """<?xml version="1.0" ?>
<!-- one CA-solved microbe on material 3, no kinetics: the biomass only moves -->
<parameters>
    <path><input_path>input</input_path><output_path>output</output_path></path>
    <simulation_mode>
        <biotic_mode>true</biotic_mode>
        <enable_kinetics>{kin}</enable_kinetics>
    </simulation_mode>
    <LB_numerics>
        <domain>
            <nx>{nx}</nx><ny>{ny}</ny><nz>{nz}</nz>
            <dx>10</dx><unit>um</unit>
            <characteristic_length>80</characteristic_length>
            <filename>geometry.dat</filename>
            <material_numbers><pore>2</pore><solid>0</solid><bounce_back>1</bounce_back><microbe0>3</microbe0></material_numbers>
        </domain>
        <delta_P>0</delta_P>
        <Peclet>0</Peclet>
        <tau>0.8</tau>
        <iteration>
            <ade_max_iT>{steps}</ade_max_iT>
            <ade_update_interval>1</ade_update_interval>
        </iteration>
    </LB_numerics>
    <chemistry>
        <number_of_substrates>1</number_of_substrates>
        <substrate0>
            <name_of_substrates>A</name_of_substrates>
            <initial_concentration>0.1</initial_concentration>
            <substrate_diffusion_coefficients><in_pore>1e-9</in_pore><in_biofilm>2e-10</in_biofilm></substrate_diffusion_coefficients>
            <left_boundary_type>Dirichlet</left_boundary_type><left_boundary_condition>1.0</left_boundary_condition>
            <right_boundary_type>Neumann</right_boundary_type><right_boundary_condition>0</right_boundary_condition>
        </substrate0>
    </chemistry>
    <microbiology>
        <number_of_microbes>1</number_of_microbes>
        <thrd_biofilm_fraction>0.1</thrd_biofilm_fraction>
        {bmax}
        <CA_method>{method}</CA_method>
        <ca_seed>99</ca_seed>
        <microbe0>
            <name_of_microbes>B</name_of_microbes>
            <solver_type>CA</solver_type>
            <initial_densities>{b0}</initial_densities>
            <decay_coefficient>0</decay_coefficient>
        </microbe0>
    </microbiology>
</parameters>
"""


def write_ca_case(tmp, mask, steps=6, method="fraction", b0=3.0, bmax=1.0, kinetics=False):
    nx, ny, nz = mask.shape
    os.makedirs(os.path.join(tmp, "input"), exist_ok=True)
    xml = os.path.join(tmp, "CompLaB.xml")
    bm = "" if bmax is None else "<maximum_biomass_density>%r</maximum_biomass_density>" % bmax
    open(xml, "w").write(CA_CASE.format(nx=nx - 2, ny=ny, nz=nz, steps=steps, method=method, b0=b0, bmax=bm,
                                        kin="true" if kinetics else "false"))
    with open(os.path.join(tmp, "input", "geometry.dat"), "w") as f:
        for x in range(1, nx - 1):
            f.write("\n".join(str(int(v)) for v in mask[x].reshape(-1)) + "\n")
    return xml


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
def test_print_config_cellular_automaton(tmp_path):
    import numpy as np
    mask = np.full((12, 8, 8), 2, np.uint8)
    mask[5, 4, 4] = 3
    xml = write_ca_case(str(tmp_path), mask, method="half")
    c = json.loads(subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True, check=True).stdout)
    assert c["ca_enabled"] == 1 and c["ca_half"] == 1
    assert c["ca_bmax"] == 1.0 and c["ca_thrd_frac"] == 0.1 and c["ca_seed"] == 99
    assert c["microbe_code"] == [3] and c["bio"] == [3]
    assert c["ns_update_interval"] == 1 and c["ade_update_interval"] == 1
    # complab_functions.hh:1175-1186: Bmax is required for a single CA microbe,
    # CA_method must be half or fraction
    xml = write_ca_case(str(tmp_path), mask, bmax=None)
    r = subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1 and "maximum_biomass_density" in r.stderr
    xml = write_ca_case(str(tmp_path), mask, method="quarter")
    r = subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True)
    assert r.returncode == 1 and "CA_method" in r.stderr


EQ_BLOCK = """    <equilibrium>
        <enabled>true</enabled>
        <components>A</components>
        <stoichiometry><species0>1</species0><species1>0</species1></stoichiometry>
        <logK><species0>0</species0><species1>0</species1></logK>
        {solver}
    </equilibrium>
</parameters>
"""


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
@pytest.mark.parametrize("xml_solver,flag,want", [("", None, "newton"), ("<solver>pcf</solver>", None, "pcf"),
                                                  ("<solver>PCF</solver>", "newton", "newton"),
                                                  ("", "pcf", "pcf")])
def test_equilibrium_solver_choice(tmp_path, xml_solver, flag, want):
    """<equilibrium><solver> (extension) and --eq-solver pick the transport
    step's speciation: Newton by default, the reference's PCF + Anderson on
    request; the command line wins."""
    xml = write_case(str(tmp_path))
    text = open(xml).read().replace("</parameters>\n", EQ_BLOCK.format(solver=xml_solver))
    open(xml, "w").write(text)
    cmd = [DRIVER, xml, "--print-config"] + (["--eq-solver", flag] if flag else [])
    c = json.loads(subprocess.run(cmd, capture_output=True, text=True, check=True).stdout)
    assert c["use_equilibrium"] == 1 and c["eq_solver"] == want
    open(xml, "w").write(text.replace(xml_solver, "<solver>anderson</solver>") if xml_solver else text)
    if xml_solver:
        r = subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True)
        assert r.returncode == 1 and "solver" in r.stderr


def _ref_examples():
    from conftest import reference_root
    root = reference_root()
    return os.path.join(root, "examples") if root else None
SUPPORTED = ["01_flow_only", "02_diffusion_only", "03_abiotic_kinetics", "04_equilibrium",
             "05_biotic_cellular_automaton", "06_biotic_finite_difference", "07_biotic_lattice_boltzmann",
             "08_two_microbes", "11_surrogate", "13_precipitation", "14_dissolution", "15_precip_and_dissolution"]


def _net_args(d):
    # example 11's network, which the reference compiles in, as the driver's file
    return ["--surrogate", "shipped_network.txt"] if os.path.exists(os.path.join(d, "shipped_network.txt")) else []


def _example_xml(name):
    # the supported examples travel as fixtures (tests/golden/examples)
    fx = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "examples", name)
    if os.path.isdir(fx):
        return fx, "CompLaB.xml"
    ex = _ref_examples()
    d = os.path.join(ex, name) if ex else ""
    if not ex or not os.path.isdir(d):
        pytest.skip("reference examples absent")
    xs = sorted(f for f in os.listdir(d) if f.endswith(".xml"))
    assert xs, name
    return d, xs[0]


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
@pytest.mark.parametrize("name", SUPPORTED)
def test_reference_example_configs_parse(name):
    """The reference's own example inputs (CPU, when the reference tree is
    present): the driver reads each CompLaB.xml of the examples whose
    reaction types this library implements, in the reference's schema."""
    d, xml = _example_xml(name)
    r = subprocess.run([DRIVER, xml, "--print-config"] + _net_args(d), cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = json.loads(r.stdout)
    assert c["nx"] >= 3 and c["ny"] >= 1 and c["nz"] >= 1
    assert len(c["names"]) >= 1
    if name == "04_equilibrium":
        assert c["use_equilibrium"] == 1 and c["n_comp"] >= 1
    if name in ("13_precipitation", "15_precip_and_dissolution"):
        assert c["precip_enabled"] == 1
    if name in ("14_dissolution", "15_precip_and_dissolution"):
        assert c["dissol_enabled"] == 1 and c["n_phases"] >= 1
    if name == "05_biotic_cellular_automaton":
        assert c["ca_enabled"] == 1


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
def test_finite_difference_biomass_config(tmp_path):
    """Example 06's finite-difference microbe: the driver reads it as sessile
    biomass with the CA's mask state, reports the microbe as FD and nu / refNu
    of its step (microbe 0's biomass over the first solute's pore
    diffusion); without the biomass diffusion coefficients it refuses the
    input, as the reference does (complab_functions.hh:1128)."""
    d, xml = _example_xml("06_biotic_finite_difference")
    r = subprocess.run([DRIVER, xml, "--print-config"], cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = json.loads(r.stdout)
    assert c["fd"] == [1] and c["ca_enabled"] == 1
    assert c["fd_nu_ratio"] == pytest.approx(3e-13 / 5e-10)
    import shutil
    e = tmp_path / "ex"
    shutil.copytree(d, e)
    x = (e / xml).read_text()
    a0, a1 = x.index("<biomass_diffusion_coefficients>"), x.index("</biomass_diffusion_coefficients>")
    (e / xml).write_text(x[:a0] + x[a1 + len("</biomass_diffusion_coefficients>"):])
    r = subprocess.run([DRIVER, xml, "--print-config"], cwd=e, capture_output=True, text=True)
    assert r.returncode == 1 and "Finite Difference" in r.stderr


@pytest.mark.skipif(not driver_available(), reason="host driver not built")
@pytest.mark.parametrize("name", SUPPORTED)
def test_example_rate_tables_and_config_dump(name, tmp_path):
    """Each example fixture with its rates.xml (the table form of the rate law
    the reference compiles in): the driver loads the table, and --dump-config
    writes the parsed cl_config, byte for byte the size of the ABI struct,
    with the geometry beside it (no GPU needed in --print-config mode)."""
    import numpy as np
    from conftest import load_pkg
    pkg = load_pkg()
    d, xml = _example_xml(name)
    args = [DRIVER, xml, "--print-config", "--dump-config", str(tmp_path / "c.bin")] + _net_args(d)
    if os.path.exists(os.path.join(d, "rates.xml")):
        args[2:2] = ["--rates", "rates.xml"]
    r = subprocess.run(args, cwd=d, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = json.loads(r.stdout)
    raw = open(tmp_path / "c.bin", "rb").read()
    assert len(raw) == ctypes_sizeof(pkg.Config)
    cfg = pkg.Config.from_buffer_copy(raw)
    assert (cfg.nx, cfg.ny, cfg.nz) == (c["nx"], c["ny"], c["nz"])
    mask = np.fromfile(tmp_path / "c.bin.mask", np.uint8)
    assert mask.size == cfg.nx * cfg.ny * cfg.nz
    want_rxn = {"03_abiotic_kinetics": 1, "05_biotic_cellular_automaton": 1, "06_biotic_finite_difference": 1,
                "07_biotic_lattice_boltzmann": 1,
                "08_two_microbes": 2, "13_precipitation": 1, "15_precip_and_dissolution": 1}.get(name, 0)
    assert cfg.n_rxn == want_rxn
    if name == "05_biotic_cellular_automaton":
        assert cfg.decay[0] == 1e-6 and cfg.rxn[0].monod_ks[0] == 5e-2 and cfg.rxn[0].nu[0] == -2.5
    if name in ("14_dissolution", "15_precip_and_dissolution"):
        assert cfg.n_phases == 1 and cfg.phases[0].k > 0 and cfg.phases[0].n_mass == 1
    # an LBM-solved microbe is carried by one more mobile solute named after it
    if name == "07_biotic_lattice_boltzmann":
        assert cfg.n_solutes == 3 and cfg.microbe_carrier[0] == 3 and c["names"][2] == "Bug"
        assert cfg.ca_enabled == 0 and cfg.c0[2] == 1.0
    if name == "08_two_microbes":
        assert cfg.microbe_carrier[0] == 0 and cfg.microbe_carrier[1] == 3 and cfg.ca_enabled == 1
        assert cfg.microbe_code[0] == 3 and cfg.microbe_code[1] == 0


def ctypes_sizeof(t):
    import ctypes
    return ctypes.sizeof(t)
