"""GPU against the FP64 oracle on the benchmark configurations themselves.

Each case runs a configuration as its benchmark states it (the coupled one
on a 128x64x64 sample; step counts reduced only where the oracle's run time
on the host cores forces it) and reports the relative L2 error of every
field against the step count.  With COMPLAB_PARITY_LOG set to a file name the
tables are appended there as JSON lines.

Tolerances (FP32 populations against the FP64 oracle):
  64^3 flow, 2000 steps: velocity rel. L2 <= 1e-4;
  its breakthrough curves (1000 transport steps; the plane-mean concentration
  at x = 8 and at the outlet plane every 10 steps): rel. L2 <= 1e-4 at x = 8,
  every sample of both within 1e-5 absolute;
  transport with reactions: concentrations rel. L2 <= 1e-4, biomass <= 1e-5;
  masks after node conversion and the conversion counts: bit-exact.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def log(case, table):
    path = os.environ.get("COMPLAB_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"case": case, "table": table}) + "\n")


def test_flow_transport_64cubed_as_stated(gpu_lib, pkg, wl):
    """64^3 voxels (plus the two boundary planes), spheres r 4-8 to porosity
    0.40, rho 1.001 / 1.000, tau 0.8, 2000 flow steps; then one solute, tau
    0.7, C = 1 Dirichlet inlet, zero-gradient outlet, C = 0 initially, 1000
    steps.  The oracle runs its own flow, so the transport comparison carries
    the flow's error too."""
    nx, ny, nz = 66, 64, 64
    mask = wl.sphere_pack(nx, ny, nz, 0.40, 4.0, 8.0, seed=101)
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0,
                          solutes=[{"tau": 0.7, "c0": 0.0, "left": "D", "left_value": 1.0, "right": "N"}])
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    fl = o.Flow(cfg, mask)
    table = []
    for k in range(4):
        lat.flow_steps(500)
        fl.step(500)
        ug = np.stack([lat.field(pkg.FIELD_FLOW_U, c).reshape(-1) for c in range(3)])
        _, uo = fl.macro()
        table.append({"flow_step": 500 * (k + 1), "u_rel_l2": rel_l2(ug, uo)})
    lat.couple_velocity()
    lat.ade_init()
    _, uo = fl.macro()
    tr = o.Transport(cfg, mask, u=uo)
    bg, bo, mg, mo = [], [], [], []
    for k in range(100):
        lat.step(10)
        tr.step(10)
        cg = lat.field(pkg.FIELD_CONC, 0).reshape(nx, ny, nz)
        co = tr.density(0).reshape(nx, ny, nz)
        bg.append(cg[nx - 2].mean())
        bo.append(co[nx - 2].mean())
        mg.append(cg[8].mean())
        mo.append(co[8].mean())
        if (k + 1) % 25 == 0:
            table.append({"ade_step": 10 * (k + 1), "c_rel_l2": rel_l2(cg, co),
                          "breakthrough_x8_rel_l2": rel_l2(mg, mo), "outlet_mean_gpu": float(bg[-1]),
                          "outlet_mean_oracle": float(bo[-1])})
    log("C1 64^3 flow + transport", table)
    assert table[3]["u_rel_l2"] <= 1e-4, table
    assert table[-1]["c_rel_l2"] <= 1e-4, table
    assert rel_l2(mg, mo) <= 1e-4
    assert np.max(np.abs(np.array(mg) - np.array(mo))) <= 1e-5
    assert np.max(np.abs(np.array(bg) - np.array(bo))) <= 1e-5
    assert mo[-1] > 0.05          # the front has passed x = 8
    lat.close()


def test_biotic_ca_128cubed(gpu_lib, pkg, wl):
    """128^3 sphere pack (porosity 0.35, radii 5-10, walled duct), four
    solutes with dual-Monod kinetics and the CA biofilm; biomass seeded at
    10-50 on 2% of the wall-adjacent pore voxels, then scaled so that colonies
    exceed Bmax and the CA spreads them; 50 steps of transport + CA block.
    The velocity is the GPU's (the 64^3 case pins the flow)."""
    n = 128
    mask = wl.walled_pack(n, n, n, 0.35, 5.0, 10.0, seed=21)
    cfg = wl.biotic_config(pkg, n, n, n)
    bio = wl.seed_biomass(mask, 22) * 3.0
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(300)
    lat.couple_velocity()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)])
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
    tr = o.Transport(cfg, mask, u=u)
    tr.set_biomass(0, bio)
    tr.ca_init()
    assert lat.ca_update_mask() == tr.ca_update_mask()
    table = []
    sweeps_g = sweeps_o = 0
    for step in range(1, 51):
        lat.step(1)
        tr.step(1)
        g = lat.ca_redistribute()
        r = tr.ca_redistribute()
        sweeps_g += g[1]
        sweeps_o += r[1]
        if step in (1, 10, 25, 50):
            row = {"step": step, "mask_diff": int((lat.mask().reshape(-1) != tr.mask).sum()),
                   "bio_rel_l2": rel_l2(lat.field(pkg.FIELD_BIOMASS, 0).reshape(-1), tr.biomass(0)),
                   "sweeps_gpu": sweeps_g, "sweeps_oracle": sweeps_o}
            for s in range(4):
                row["c%d_rel_l2" % s] = rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), tr.density(s))
            table.append(row)
    log("C2 128^3 biotic + CA", table)
    last = table[-1]
    assert sweeps_o > 0 and sweeps_g == sweeps_o
    assert last["mask_diff"] == 0
    assert last["bio_rel_l2"] <= 1e-5
    for s in range(4):
        assert last["c%d_rel_l2" % s] <= 1e-4, s
    lat.close()


def test_surrogate_64cubed_sample(gpu_lib, pkg, wl):
    """The surrogate-rate workload (porosity 0.4, two organisms with
    3 -> 20 -> 20 -> 4 networks, six solutes) on a 64^3 sample, 200 steps."""
    nx, ny, nz = 66, 64, 64
    mask = wl.sphere_pack(nx, ny, nz, 0.40, 4.0, 8.0, seed=31)
    cfg = wl.surrogate_config(pkg, nx, ny, nz)
    nets = wl.surrogate_nets(pkg)
    b0 = wl.seed_biomass(mask, 32, frac=0.3, lo=0.005, hi=0.05)
    b1 = wl.seed_biomass(mask, 33, frac=0.3, lo=0.005, hi=0.05)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(300)
    lat.couple_velocity()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)])
    for slot in range(2):
        lat.set_surrogate(slot, nets[slot])
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, b0)
    lat.set_field(pkg.FIELD_BIOMASS, 1, b1)
    tr = o.Transport(cfg, mask, u=u)
    tr.set_surrogates(nets)
    tr.set_biomass(0, b0)
    tr.set_biomass(1, b1)
    table = []
    for k in range(4):
        lat.step(50)
        tr.step(50)
        row = {"step": 50 * (k + 1)}
        for s in range(6):
            row["c%d_rel_l2" % s] = rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), tr.density(s))
        for m in range(2):
            row["b%d_rel_l2" % m] = rel_l2(lat.field(pkg.FIELD_BIOMASS, m).reshape(-1), tr.biomass(m))
        table.append(row)
    log("C4 surrogate 64^3 sample", table)
    last = table[-1]
    for s in range(6):
        assert last["c%d_rel_l2" % s] <= 1e-4, (s, table)
    for m in range(2):
        assert last["b%d_rel_l2" % m] <= 1e-5, (m, table)
    lat.close()


def test_coupled_128x64x64_sample_with_node_conversion(gpu_lib, pkg, wl):
    """The coupled workload (porosity 0.35, radii 5-10; flow + 8 mobile
    solutes + mineral; dual Monod, saturation-driven surface precipitation,
    3-component Newton every step) on a 128x64x64 sample for 200 steps.  Part
    of the wall-adjacent voxels start with a mineral inventory below the
    conversion threshold, so node conversions happen at steps 100 and 200: the
    masks and counts must agree exactly.  After each conversion the GPU
    switches the dynamics, re-solves the flow and re-couples the velocity,
    which the oracle's transport then takes."""
    nx, ny, nz = 128, 64, 64
    mask = wl.sphere_pack(nx, ny, nz, 0.35, 5.0, 10.0, seed=41)
    cfg = wl.coupled_config(pkg, nx, ny, nz)
    cfg.max_precip_rho = 1e-3
    bio = wl.seed_biomass(mask, 42)
    mineral = wl.seed_mineral(mask, 43, cfg.max_precip_rho)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(300)
    lat.couple_velocity()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)])
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
    lat.set_field(pkg.FIELD_CONC, 8, mineral)
    tr = o.Transport(cfg, mask, u=u)
    tr.set_biomass(0, bio)
    tr.set_conc(8, mineral)
    table = []
    changes = []
    for k in range(2):
        assert lat.step(100) == pkg.OK
        assert tr.step(100) == 0
        cg = lat.precip_convert()
        co = tr.precip_convert()
        changes.append((cg, co))
        np.testing.assert_array_equal(lat.mask().reshape(-1), tr.mask)
        lat.update_dynamics()
        lat.flow_steps(100)
        lat.couple_velocity()
        tr.u[:] = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)]).reshape(-1)
        row = {"step": 100 * (k + 1), "converted_gpu": cg, "converted_oracle": co}
        for s in range(cfg.n_solutes):
            row["c%d_rel_l2" % s] = rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), tr.density(s))
        row["bio_rel_l2"] = rel_l2(lat.field(pkg.FIELD_BIOMASS, 0).reshape(-1), tr.biomass(0))
        table.append(row)
    log("C5 coupled 128x64x64 sample", table)
    assert all(cg == co for cg, co in changes) and changes[0][0] > 0, changes
    last = table[-1]
    for s in range(cfg.n_solutes):
        assert last["c%d_rel_l2" % s] <= 1e-4, (s, table)
    assert last["bio_rel_l2"] <= 1e-5
    lat.close()
