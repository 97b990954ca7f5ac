"""The oracle against the committed golden fixtures made from the reference's
own code (tests/golden/make_golden.py).  CPU only; no reference tree needed."""
import os

import numpy as np
import pytest

from oracle import oracle as o

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def shipped_net(pkg):
    z = np.load(os.path.join(GOLD, "surrogate_shipped.npz"))
    W = [z["W%d" % l] for l in range(5)]
    b = [z["b%d" % l] for l in range(5)]
    widths = [W[0].shape[1]] + [w.shape[0] for w in W]
    net = pkg.make_surrogate_net(widths, W, b, z["x_offset"], z["x_gain"], [float(z["y_offset"])],
                                 [float(z["y_gain"])], x_ymin=float(z["x_ymin"]), y_ymin=float(z["y_ymin"]))
    return net, z


def test_oracle_surrogate_matches_shipped_reference(pkg):
    """verifyExport.py's bar: <= 1e-10 relative on the exported network."""
    net, z = shipped_net(pkg)
    y = o.surrogate_forward(net, z["fin"])[:, 0]
    y = np.where(y < 1e-8, 0.0, y)     # the shipped model's dust clamp (surrogateModel.hh:429)
    ref = z["bior"]
    np.testing.assert_allclose(y, ref, rtol=1e-10, atol=1e-14)


def test_oracle_newton_matches_pcf_fixture(pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, z["S"], z["logk"], list(z["comp_species"]), max_iter=200, tol=1e-10)
    S, logk, T = z["S"], z["logk"], z["totals"]
    from conftest import load_workloads
    wl = load_workloads()
    x, it, st = o.eq_batch(sys_, T, wl.cold_species(S, T, list(z["comp_species"])), start=0)
    assert (st == 0).all()
    c = 10 ** (logk[None, :] + x @ S.T)
    ok = z["pcf_cv"] == 1
    big = c > 1e-25
    rel = np.abs(z["pcf_out"] - c) / c
    assert np.median(rel[ok[:, None] & big]) < 1e-8
    np.testing.assert_allclose(x, z["xstar"], atol=1e-7)


def test_carbonate_fixture(pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, z["S4"], z["logk4"], [0, 1], max_iter=100, tol=1e-12)
    sp = z["species4"]
    T = np.maximum(np.clip(sp, 1e-30, 10) @ z["S4"], 1e-30)
    x, it, st = o.eq_batch(sys_, T, sp, start=0)
    assert (st == 0).all()
    c = 10 ** (z["logk4"][None, :] + x @ z["S4"].T)
    np.testing.assert_allclose(c, z["out4"], rtol=1e-6)
