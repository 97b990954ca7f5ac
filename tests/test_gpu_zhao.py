"""The reference's default rate laws (the Zhao uranium / iron / sulfur
network) compiled into the transport step (cl_config.rate_law =
CL_RATELAW_ZHAO) against the FP64 oracle driven by the same laws built for
the host (oracle/libratelaw_host.so, pinned to the reference's own headers by
tests/test_ratelaw_port.py).

24 substrates (15 mobile), 12 biomass pools held as sessile fields, dt equal
to the laws' stability time step (1e-4 s, as their header requires), suspended
pools large enough that their rates pass the 1e-12 increment gate.
Tolerances: concentrations rel. L2 <= 1e-4, biomass <= 1e-5 (as for the
table-driven chemistries)."""
import ctypes
import os

import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
IMMOBILE = (2, 4, 5, 6, 9, 13, 21, 22, 23)


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def zhao_config(pkg, nx, ny, nz):
    c0 = np.full(24, 1e-3)
    c0[[1, 3, 8]] = [1e-5, 1e-3, 1e-3]          # U(VI), Fe(II), sulfide
    c0[[2, 12, 13]] = 0.0                        # U(IV), methane, S0 start empty
    c0[[4, 5, 6]] = 1e-2                         # Fe(III) easy / medium / hard
    c0[9] = 1e-4                                 # FeS
    c0[10], c0[11] = 2e-3, 1e-7                  # bicarbonate, H+
    c0[[21, 22, 23]] = 1e-4                      # surface sites
    sol = []
    for s in range(24):
        if s in IMMOBILE:
            sol.append({"immobile": True, "c0": float(c0[s])})
        else:
            sol.append({"tau": 0.8, "c0": float(c0[s]), "left": "D", "left_value": float(c0[s]), "right": "N"})
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0, solutes=sol, microbes=12, dt=1e-4)
    cfg.rate_law = pkg.RATELAW_ZHAO
    cfg.enable_kinetics = 1
    cfg.enable_abiotic = 1
    return cfg


def test_zhao_network_in_the_step(gpu_lib, pkg, wl):
    mask = wl.sphere_pack(20, 12, 12, 0.5, 2.0, 3.0, seed=61)
    nx, ny, nz = mask.shape
    cfg = zhao_config(pkg, nx, ny, nz)
    rng = np.random.default_rng(62)
    pore = (mask == 2).astype(float)
    bio = []
    for m in range(12):
        suspended = m in (3, 7, 9, 11)
        scale = 5e-2 if suspended else 5e-5
        bio.append(pore * rng.uniform(0.2, 1.0, mask.shape) * scale)
    lat = pkg.Lattice(cfg)
    assert lat.get_option(pkg.OPT_COMPILED_CHEM) == pkg.CHEM_ZHAO24
    with pytest.raises(pkg.CLError):
        lat.set_option(pkg.OPT_COMPILED_CHEM, 0)      # no table form of a compiled law
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(100)
    lat.couple_velocity()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)])
    lat.ade_init()
    for m in range(12):
        lat.set_field(pkg.FIELD_BIOMASS, m, bio[m])
    port = ctypes.CDLL(os.path.join(ROOT, "oracle", "libratelaw_host.so"))
    tr = o.Transport(cfg, mask, u=u)
    tr.set_rate_law(ctypes.cast(port.port_zhao_kinetics, ctypes.c_void_p).value,
                    ctypes.cast(port.port_zhao_abiotic, ctypes.c_void_p).value)
    for m in range(12):
        tr.set_biomass(m, bio[m])
    for n in (1, 4, 25):
        assert lat.step(n) == pkg.OK
        tr.step(n)
    for s in range(24):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), tr.density(s)) < 1e-4, s
    for m in range(12):
        assert rel_l2(lat.field(pkg.FIELD_BIOMASS, m).reshape(-1), tr.biomass(m)) < 1e-5, m
    # the network did something: U(IV) and methane appear, FeS forms from Fe(II)
    # + sulfide (S0's reactions stay below the 1e-12 increment gate here)
    for s in (2, 12):
        assert tr.density(s).max() > 0.0, s
    assert lat.field(pkg.FIELD_CONC, 9).max() > 1e-4
    lat.close()


def test_zhao_needs_its_layout(gpu_lib, pkg):
    cfg = pkg.make_config(8, 4, 4, solutes=[{"tau": 0.8}] * 4, microbes=1)
    cfg.rate_law = pkg.RATELAW_ZHAO
    with pytest.raises(pkg.CLError):
        pkg.Lattice(cfg)
