"""The reference's own example inputs through the host driver on the GPU,
against the FP64 oracle replaying the same run.

Examples 07 and 08 solve a microbe by LBM (the reference's planktonic
bFree lattice): the driver carries it as one more mobile solute named after
it (cl_config.microbe_carrier), compared as a solute field.  Example 06
solves its sessile microbe by finite differences (cl_fd_diffuse between two
mask updates each step); example 11 adds the surrogate reaction type with
the network the reference compiles in (shipped_network.txt, --surrogate).

Each folder under tests/golden/examples holds one example's CompLaB.xml and
geometry exactly as the reference ships them (copied by make_examples.py)
and rates.xml, the table form of the rate law that the reference compiles in
from the example's headers.  The driver runs the example with --rates and
--dump-config; the oracle replays the run from the dumped configuration and
geometry in the driver's order (complab.cpp:560-1860 as the driver follows
it): the flow solved from rest to the driver's tolerance where a Peclet
number is set (the calibrated pressure drop is in the dump), then per step
the transport step, the cellular-automaton block with its dynamics switch,
and the precipitation and dissolution node conversions on their intervals.
Under flow, a node conversion or a CA mask change re-solves the flow, which
the oracle's transport does not replay: such a run is compared at the step of
its first conversion.

Tolerances (FP32 populations against FP64, as the other transport tests):
solute fields relative L2 <= 1e-4, and <= 3e-4 for a lattice relaxing at
omega > 1.99 (example 08's LBM-solved microbe, tau 0.50018: the FP64 oracle
itself amplifies a one-ulp FP32 rounding of that lattice eighteenfold in 300
steps, test_oracle_carrier_sensitivity.py; the GPU's FP32 populations round
every step and it ends 1.1e-4 from the oracle after 1000 steps, while that
run's donor and product stay within 5e-6); biomass relative L2 <= 1e-5; conversion
counts and masks equal up to voxels within the transport tolerance of a
threshold (at most 2, or 2% of the changes); the flow solve's iteration count
within 2% of the oracle's.
"""
import json
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import oracle as o
from test_driver_config import DRIVER

pytestmark = pytest.mark.gpu

EXAMPLES = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "examples")
# example: transport steps (the example's own ade_max_iT)
CASES = {"01_flow_only": 400, "02_diffusion_only": 2000, "03_abiotic_kinetics": 1500, "04_equilibrium": 600,
         "05_biotic_cellular_automaton": 1000, "06_biotic_finite_difference": 1000,
         "07_biotic_lattice_boltzmann": 1000, "08_two_microbes": 1000, "11_surrogate": 500,
         "13_precipitation": 2000, "14_dissolution": 2000, "15_precip_and_dissolution": 3000}
# Example 08 runs without flow: its LBM-solved microbe diffuses at 3e-13 m^2/s,
# so its lattice relaxes at tau = 0.5002, and under the example's Pe = 1 flow
# (up to u = 0.14, a grid Peclet number of ~3000) BGK advection-diffusion is
# unstable: the oracle and the GPU both see that microbe's density climb from
# 1.03 to 1.35 within 40 steps of a uniform 1.0.  The CA and both microbes'
# kinetics run as the example states them.
EDITS = {"08_two_microbes": [("<Peclet>1</Peclet>", "<Peclet>0</Peclet>")]}


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def stage(name, tmp):
    d = os.path.join(str(tmp), name)
    shutil.copytree(os.path.join(EXAMPLES, name), d)
    if name in EDITS:
        x = open(os.path.join(d, "CompLaB.xml")).read()
        for old, new in EDITS[name]:
            assert old in x
            x = x.replace(old, new)
        open(os.path.join(d, "CompLaB.xml"), "w").write(x)
    return d


def driver(d, *args):
    cmd = [DRIVER, "CompLaB.xml"] + (["--rates", "rates.xml"] if os.path.exists(os.path.join(d, "rates.xml")) else [])
    if os.path.exists(os.path.join(d, "shipped_network.txt")):
        cmd += ["--surrogate", "shipped_network.txt"]
    return subprocess.run(cmd + list(args), cwd=d, capture_output=True, text=True)


def load_net(pkg, path):
    """A driver network file (--surrogate) as the library's cl_surrogate_net."""
    kv, key = {}, None
    for line in open(path):
        for tok in line.split("#")[0].split():
            try:
                v = float(tok)
            except ValueError:
                key = tok
                kv[key] = []
                continue
            kv[key].append(v)
    L = int(kv["layers"][0])
    widths = [int(w) for w in kv["widths"]]
    W = [np.array(kv["W%d" % l]).reshape(widths[l + 1], widths[l]) for l in range(L)]
    b = [np.array(kv["b%d" % l]) for l in range(L)]
    return pkg.make_surrogate_net(widths, W, b, kv["x_offset"], kv["x_gain"], kv["y_offset"], kv["y_gain"],
                                  x_ymin=kv["x_ymin"][0], y_ymin=kv["y_ymin"][0])


def solute_switch(tr):
    """updateSoluteDynamics3D on the oracle's classes after a CA mask change."""
    wall = (tr.mask == 0) | (tr.mask == 1)
    pore = np.isin(tr.mask, [tr.cfg.pore_codes[i] for i in range(tr.cfg.n_pore_codes)])
    tr.ade[~wall & pore] = 2
    tr.ade[~wall & ~pore] = 3


def replay(pkg, cj, cfg, mask, steps, d=None):
    """The oracle's run of the driver's loop; returns the transport state, the
    event counts, the step the comparison stops at and the flow iterations."""
    flow = cj["Pe"] > 1e-12
    u, flow_it = None, 0
    if flow:
        fl = o.Flow(cfg, mask)
        flow_it, _ = fl.solve(int(cj["ns_max_iT1"]), cj["ns_converge_iT1"])
        _, u = fl.macro()
    tr = o.Transport(cfg, mask, u=u)
    if cfg.n_srg:
        tr.set_surrogates([load_net(pkg, os.path.join(d, f)) for f in cj["surrogate_files"]])
    for m in range(cfg.n_microbes):
        if cfg.microbe_carrier[m]:
            continue                      # LBM-solved: its carrier solute's c0
        b = np.zeros(mask.size)
        for mat, b0 in zip(cj["bio_materials"][m], cj["b0"][m]):
            b[mask == mat] = b0
        tr.set_biomass(m, b)
    ev = {"precip": 0, "dissol": 0, "ca_sweeps": 0, "ca_changes": 0}
    # finite-difference microbes: the mask update, one diffusion step with
    # nu = bioNUinPore[0] (refNu from the first solute's pore relaxation), the
    # mask update (complab.cpp:1716-1731)
    fd_bits = sum(1 << m for m, f in enumerate(cj.get("fd", [])) if f)
    fd_nu = (1.0 / cfg.omega_pore[0] - 0.5) / 4.0 * cj.get("fd_nu_ratio", 0.0)
    if cfg.ca_enabled:
        tr.ca_init()
        ch = tr.ca_update_mask()
        ev["ca_changes"] += ch
        if ch:
            solute_switch(tr)
    stop = steps
    for it in range(steps):
        tr.step(1)
        ca_resolve = False
        if cfg.ca_enabled and fd_bits:
            ch = tr.ca_update_mask()
            tr.fd_diffuse(fd_nu, fd_bits)
            ch += tr.ca_update_mask()
            ev["ca_changes"] += ch
        elif cfg.ca_enabled:
            st, sw, ch, _ = tr.ca_redistribute()
            assert st == 0
            ev["ca_sweeps"] += sw
            ev["ca_changes"] += ch
            if ch and (it % cj["ade_update_interval"] == 0 or it % cj["ns_update_interval"] == 0):
                solute_switch(tr)
            if ch and it % cj["ns_update_interval"] == 0:
                ca_resolve = True            # under flow the driver re-solves it here
        changed = 0
        if cfg.precip_enabled and it % cj["precip_interval"] == 0:
            ch = tr.precip_convert()
            ev["precip"] += ch
            changed += ch
        if cfg.dissol_enabled and it % cj["dissol_interval"] == 0:
            ch = tr.dissol_convert()
            ev["dissol"] += ch
            changed += ch
        if flow and (changed or ca_resolve):
            stop = it + 1
            break
    return tr, ev, stop, flow_it


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_example_against_oracle(gpu_lib, pkg, tmp_path, name):
    d = stage(name, tmp_path)
    cj = json.loads(driver(d, "--print-config").stdout)
    steps = CASES[name]
    assert steps == cj["ade_max_iT"]
    # the dump comes from a run of the driver itself (the flow and its
    # calibration on the GPU), one step long
    r = driver(d, "--steps", "1", "--dump-config", "run.cfg", "--quiet")
    assert r.returncode == 0, r.stderr
    cfg = pkg.Config.from_buffer_copy(open(os.path.join(d, "run.cfg"), "rb").read())
    mask = np.fromfile(os.path.join(d, "run.cfg.mask"), np.uint8)
    tr, ev, stop, flow_it = replay(pkg, cj, cfg, mask, steps, d)
    r = driver(d, "--steps", str(stop), "--quiet")
    assert r.returncode == 0, r.stderr
    out = json.loads(r.stdout.strip().splitlines()[-1])
    assert out["steps"] == stop
    if cj["Pe"] > 1e-12:
        assert abs(out["ns_iters"] - flow_it) <= max(2, 0.02 * flow_it), (out["ns_iters"], flow_it)
    od = os.path.join(d, "output")
    table = {"steps": stop}
    for s, nm in enumerate(cj["names"]):
        g = np.fromfile(os.path.join(od, "%s_%d.raw" % (nm, stop)), np.float64)
        table[nm] = rel_l2(g, tr.density(s))
    for m, nm in enumerate(cj["microbe_names"]):
        if cfg.microbe_carrier[m]:
            continue                      # compared as its carrier solute
        g = np.fromfile(os.path.join(od, "%s_%d.raw" % (nm, stop)), np.float64)
        table["biomass " + nm] = rel_l2(g, tr.biomass(m))
    for key in ("precip", "dissol"):
        got = out["%s_changes" % key]
        assert abs(got - ev[key]) <= max(2, ev[key] // 50), (key, got, ev[key])
    m_g = np.fromfile(os.path.join(od, "mask_%d.u8" % stop), np.uint8)
    changed = int((tr.mask != mask).sum())
    assert int((m_g != tr.mask).sum()) <= max(2, changed // 50), (int((m_g != tr.mask).sum()), changed)
    if cfg.ca_enabled:
        assert out["ca_sweeps"] == ev["ca_sweeps"] and out["ca_mask_changes"] == ev["ca_changes"]
    for s, nm in enumerate(cj["names"]):
        tol = 3e-4 if max(cfg.omega_pore[s], cfg.omega_bio[s]) > 1.99 else 1e-4
        assert table[nm] <= tol, (nm, table)
    for m, nm in enumerate(cj["microbe_names"]):
        if not cfg.microbe_carrier[m]:
            assert table["biomass " + nm] <= 1e-5, (nm, table)
