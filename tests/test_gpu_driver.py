"""The host driver end to end on the GPU: CompLaB.xml in, fields out, against
the FP64 oracle stepped in the same order (the same tolerances as the other
transport tests), and the Peclet calibration of the flow."""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as o
from test_driver_config import DRIVER, write_case

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
