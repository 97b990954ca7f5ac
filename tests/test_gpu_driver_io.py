"""The host driver's checkpoint and VTI output on the GPU, on the reference's
example 13 (flow at Pe 1, FeS precipitation whose first node conversion, at
step 1500, re-solves the flow).

  - a run of 1600 steps saving a checkpoint every 800 steps, and a second run
    restarted from the checkpoint of step 800: every final field bit for bit
    equal (the restart crosses the conversion and its flow re-solve);
  - the VTI files of the final step hold the same values as the raw arrays
    (Density of each solute over the interior planes, FP64), the material
    numbers, and nsLattice's velocity (FP32) and its norm.
"""
import base64
import json
import os
import re
import shutil
import subprocess
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from test_driver_config import DRIVER

pytestmark = pytest.mark.gpu
EX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "examples", "13_precipitation")


def stage(tmp, name, vtk, chk):
    d = os.path.join(str(tmp), name)
    shutil.copytree(EX, d)
    x = open(os.path.join(d, "CompLaB.xml")).read()
    x = re.sub(r"<save_VTK_interval>[^<]*</save_VTK_interval>", "<save_VTK_interval>%d</save_VTK_interval>" % vtk, x)
    x = re.sub(r"<save_CHK_interval>[^<]*</save_CHK_interval>", "<save_CHK_interval>%d</save_CHK_interval>" % chk, x)
    open(os.path.join(d, "CompLaB.xml"), "w").write(x)
    return d


def run(d, *args):
    r = subprocess.run([DRIVER, "CompLaB.xml", "--rates", "rates.xml", "--quiet"] + list(args), cwd=d,
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout.strip().splitlines()[-1])


def vti_arrays(path):
    out = {}
    for da in ET.parse(path).getroot().iter("DataArray"):
        raw = base64.b64decode(da.text.strip())
        n = int(np.frombuffer(raw[:8], np.uint64)[0])
        out[da.get("Name")] = np.frombuffer(raw[8:8 + n], np.float64 if da.get("type") == "Float64" else np.float32)
    return out


def test_checkpoint_restart_and_vti(gpu_lib, tmp_path):
    steps = 1600
    a = stage(tmp_path, "a", vtk=800, chk=800)
    out_a = run(a, "--steps", str(steps))
    assert out_a["precip_changes"] > 0 and out_a["flow_resolves"] > 0
    chk = os.path.join(a, "output", "chk_800")
    meta = json.load(open(os.path.join(chk, "checkpoint.json")))
    assert meta["steps"] == 800 and meta["has_flow"] == 1
    b = stage(tmp_path, "b", vtk=800, chk=0)
    out_b = run(b, "--steps", str(steps), "--restart", chk)
    assert out_b["steps"] == steps - 800        # (its counts start at the restart)
    cj = json.loads(subprocess.run([DRIVER, "CompLaB.xml", "--rates", "rates.xml", "--print-config"], cwd=a,
                                   capture_output=True, text=True, check=True).stdout)
    nx, ny, nz = cj["nx"], cj["ny"], cj["nz"]
    for nm in cj["names"]:
        fa = np.fromfile(os.path.join(a, "output", "%s_%d.raw" % (nm, steps)), np.float64)
        fb = np.fromfile(os.path.join(b, "output", "%s_%d.raw" % (nm, steps)), np.float64)
        np.testing.assert_array_equal(fa, fb, err_msg=nm)
        # the VTI of the same step: the interior planes, x fastest
        v = vti_arrays(os.path.join(a, "output", "%s_%07d.vti" % (nm, steps)))["Density"]
        np.testing.assert_array_equal(v, fa.reshape(nx, ny, nz)[1:-1].transpose(2, 1, 0).reshape(-1))
    ma = np.fromfile(os.path.join(a, "output", "mask_%d.u8" % steps), np.uint8)
    np.testing.assert_array_equal(ma, np.fromfile(os.path.join(b, "output", "mask_%d.u8" % steps), np.uint8))
    vm = vti_arrays(os.path.join(a, "output", "maskLattice_%07d.vti" % steps))["Density"]
    np.testing.assert_array_equal(vm, ma.reshape(nx, ny, nz)[1:-1].transpose(2, 1, 0).reshape(-1).astype(float))
    ns = vti_arrays(os.path.join(a, "output", "nsLattice_%07d.vti" % steps))
    u = ns["velocity"].reshape(-1, 3)
    assert u.shape[0] == (nx - 2) * ny * nz and np.abs(u[:, 0]).max() > 0
    np.testing.assert_allclose(ns["velocityNorm"], np.sqrt((u.astype(np.float64) ** 2).sum(1)), rtol=1e-6, atol=1e-12)
    idx = json.load(open(os.path.join(a, "output", "fields.json")))
    assert any(f.endswith(".vti") for f in idx["files"])
