"""The host driver end to end on the GPU: CompLaB.xml in, fields out, against
the FP64 oracle stepped in the same order (the same tolerances as the other
transport tests), and the Peclet calibration of the flow."""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as o
from test_driver_config import DRIVER, write_case, write_ca_case

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def run_driver(xml, steps):
    r = subprocess.run([DRIVER, xml, "--steps", str(steps), "--quiet"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_driver_matches_oracle_without_flow(gpu_lib, pkg, wl, tmp_path):
    mask = wl.sphere_pack(12, 10, 10, 0.6, 1.5, 2.5, seed=41)
    nx, ny, nz = mask.shape
    xml = write_case(str(tmp_path), nx=nx - 2, ny=ny, nz=nz, Pe=0.0, dP=0.0, steps=20, mask=mask[1:-1])
    cfg_json = json.loads(subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True,
                                         check=True).stdout)
    out = run_driver(xml, 20)
    # the oracle with the driver's relaxation and time step
    om, dt = cfg_json["omega_pore"], out["dt"]
    sol = [{"tau": 1.0 / om[0], "c0": 0.1, "left": "D", "left_value": 1.0, "right": "N"},
           {"immobile": True, "c0": 0.0}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, dt=dt)
    cfg.enable_abiotic = 1
    cfg.precip_enabled = 1
    cfg.abiotic_surface_only = 1
    cfg.precip_substrate = 1
    cfg.max_precip_rho = 0.02
    cfg.precip_code = 0
    pkg.add_rxn(cfg, k=0.05, mass=[0], nu={0: -1.0, 1: 1.0})
    ref = o.Transport(cfg, mask)
    changed = 0
    for it in range(20):
        ref.step(1)
        if it % 5 == 0:
            changed += ref.precip_convert()
    # node conversion is bit-exact given the same inventories (the transport
    # tests check that); here the inventories come from FP32 transport, so a
    # voxel within the transport tolerance of the threshold may convert one
    # interval apart
    assert abs(out["precip_changes"] - changed) <= max(2, changed // 50)
    N = mask.size
    a = np.fromfile(os.path.join(str(tmp_path), "output", "A_20.raw"), np.float64)
    p = np.fromfile(os.path.join(str(tmp_path), "output", "P_20.raw"), np.float64)
    m = np.fromfile(os.path.join(str(tmp_path), "output", "mask_20.u8"), np.uint8)
    assert a.size == N and p.size == N
    assert rel_l2(a, ref.density(0)) < 1e-4
    assert rel_l2(p, ref.density(1)) < 1e-4
    assert (m != ref.mask).sum() <= max(2, int((ref.mask != mask.reshape(-1)).sum()) // 50)


def test_driver_peclet_calibration(gpu_lib, pkg, wl, tmp_path):
    mask = wl.sphere_pack(18, 12, 12, 0.55, 2.0, 3.0, seed=43)
    nx, ny, nz = mask.shape
    xml = write_case(str(tmp_path), nx=nx - 2, ny=ny, nz=nz, Pe=1.0, dP=2e-5, L=12, steps=5, mask=mask[1:-1])
    out = run_driver(xml, 5)
    assert out["ns_iters"] > 0
    # the corrected deltaP brings the outlet Darcy velocity to the target Peclet
    assert out["Pe_achieved"] == pytest.approx(1.0, rel=0.05)
    assert out["pore_mean_u"] > 0 and out["max_ux"] > 0


def ca_channel(shape, seed, n_colonies):
    """A channel with bounce-back walls on the y / z faces, 3^3 solid cubes and
    single-voxel colonies of material 3."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    mask = np.full(shape, 2, np.uint8)
    for _ in range(int(0.05 * nx * ny * nz / 27) + 1):
        x, y, z = rng.integers(1, nx - 3), rng.integers(1, ny - 3), rng.integers(1, nz - 3)
        mask[x:x + 3, y:y + 3, z:z + 3] = 0
    mask[:, 0, :] = mask[:, ny - 1, :] = 1
    mask[:, :, 0] = mask[:, :, nz - 1] = 1
    placed = 0
    while placed < n_colonies:
        x, y, z = rng.integers(2, nx - 2), rng.integers(1, ny - 1), rng.integers(1, nz - 1)
        if mask[x, y, z] == 2:
            mask[x, y, z] = 3
            placed += 1
    # the driver's inlet and outlet planes repeat the first and last slice
    mask[0], mask[-1] = mask[1], mask[-2]
    return mask


def solute_switch(ref):
    """updateSoluteDynamics3D on the oracle's classes: non-wall voxels take the
    pore or the biofilm relaxation by their mask."""
    wall = (ref.mask == 0) | (ref.mask == 1)
    pore = ref.mask == 2
    ref.ade[~wall & pore] = 2
    ref.ade[~wall & ~pore] = 3


@pytest.mark.parametrize("method", ["fraction", "half"])
def test_driver_cellular_automaton(gpu_lib, pkg, tmp_path, method):
    """Colonies seeded at 3 x Bmax spread in the first CA block after step 1;
    without kinetics nothing else moves the biomass, so biomass and mask are
    bit-exact against the oracle and the solute within the transport tolerance."""
    steps = 6
    mask = ca_channel((16, 14, 12), seed=8, n_colonies=12)
    nx, ny, nz = mask.shape
    xml = write_ca_case(str(tmp_path), mask, steps=steps, method=method, b0=3.0, bmax=1.0)
    c = json.loads(subprocess.run([DRIVER, xml, "--print-config"], capture_output=True, text=True, check=True).stdout)
    out = run_driver(xml, steps)
    assert out["ca_blocks"] >= 1 and out["ca_sweeps"] >= 1 and out["ca_mask_changes"] > 0
    sol = [{"tau": 1.0 / c["omega_pore"][0], "tau_bio": 1.0 / c["omega_bio"][0], "c0": 0.1,
            "left": "D", "left_value": 1.0, "right": "N"}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, microbes=1, pore_codes=(2,), bio_codes=(3,), dt=out["dt"])
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, 1 if method == "half" else 0, 1.0, 0.1
    cfg.microbe_code[0] = 3
    cfg.ca_seed = 99
    ref = o.Transport(cfg, mask)
    ref.set_biomass(0, np.where(mask == 3, 3.0, 0.0))
    ref.ca_init()
    if ref.ca_update_mask():
        solute_switch(ref)
    sweeps = changes = 0
    for _ in range(steps):
        ref.step(1)
        st, sw, ch, _ = ref.ca_redistribute()
        assert st == 0
        sweeps += sw
        changes += ch
        if ch:
            solute_switch(ref)
    assert out["ca_sweeps"] == sweeps and out["ca_mask_changes"] == changes
    d = str(tmp_path / "output")
    b = np.fromfile(os.path.join(d, "B_%d.raw" % steps), np.float64)
    m = np.fromfile(os.path.join(d, "mask_%d.u8" % steps), np.uint8)
    a = np.fromfile(os.path.join(d, "A_%d.raw" % steps), np.float64)
    np.testing.assert_array_equal(b, ref.biomass(0))
    np.testing.assert_array_equal(m, ref.mask)
    assert rel_l2(a, ref.density(0)) < 1e-4
