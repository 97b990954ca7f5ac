"""How sensitive the reference's example 08 is to rounding (CPU, FP64 oracle).

Its LBM-solved microbe (Bug2_efficient, carried as a solute) diffuses at
3e-13 m^2/s, so its lattice relaxes at omega = 1.99928 in the pore (tau
0.50018), within 7e-4 of BGK's stability limit: its non-equilibrium modes
decay by a factor 0.9993 a step and nothing damps a perturbation within the
run.  Two FP64 oracle runs whose carrier populations differ by one FP32 ulp
at half the sites (the rounding one step of FP32 storage makes) are stepped
300 steps: the carrier's difference grows more than tenfold while the donor,
relaxed at omega 1.25, stays at the rounding level.  FP32 populations inject
such a rounding every step, which is why the GPU-against-oracle comparison of
that field uses a looser bound than the other solutes (test_gpu_examples.py).
"""
import json
import os

import numpy as np

from oracle import oracle as o
from test_gpu_examples import EDITS, driver, rel_l2, replay, stage


def test_example_08_carrier_amplifies_one_ulp(pkg, tmp_path):
    name = "08_two_microbes"
    assert name in EDITS
    d = stage(name, tmp_path)
    cj = json.loads(driver(d, "--print-config").stdout)
    r = driver(d, "--print-config", "--dump-config", "run.cfg")
    assert r.returncode == 0, r.stderr
    cfg = pkg.Config.from_buffer_copy(open(os.path.join(d, "run.cfg"), "rb").read())
    mask = np.fromfile(os.path.join(d, "run.cfg.mask"), np.uint8)
    names = list(cj["names"])
    s_bug, s_donor = names.index("Bug2_efficient"), names.index("donor")
    assert cfg.microbe_carrier[1] == s_bug + 1
    assert 1.999 < cfg.omega_pore[s_bug] < 2.0 and abs(cfg.omega_pore[s_donor] - 1.25) < 1e-12
    N = cfg.nx * cfg.ny * cfg.nz
    a, _, _, _ = replay(pkg, cj, cfg, mask, 100)
    b, _, _, _ = replay(pkg, cj, cfg, mask, 100)
    sl = slice(s_bug * 7 * N, (s_bug + 1) * 7 * N)
    x = b.g[sl].astype(np.float32)
    rng = np.random.default_rng(8)
    pick = rng.random(x.size) < 0.5
    x[pick] = np.nextafter(x[pick], np.float32(2.0))
    b.g[sl] = x.astype(np.float64)
    d0 = rel_l2(b.density(s_bug), a.density(s_bug))
    assert 0 < d0 < 1e-7
    a.step(300)
    b.step(300)
    d_bug = rel_l2(b.density(s_bug), a.density(s_bug))
    d_donor = rel_l2(b.density(s_donor), a.density(s_donor))
    assert d_bug > 10 * d0, (d0, d_bug)
    assert d_donor < 1e-8, d_donor
