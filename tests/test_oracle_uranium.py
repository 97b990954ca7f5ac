"""The oracle's speciation on the reference's uranium tableau (17 components
over 95 species, tests/golden/uranium_tableau.npz, parsed from the
reference's own CompLaB_example_uranium_zhao.xml by make_golden.py).

  - the oracle's restatement of the reference's PCF + Anderson reproduces the
    reference's own solver compiled from its sources (recorded in the
    fixture): iterations, convergence flags and species, from the known
    species and from the cold vectors;
  - the oracle's Newton from the known answers perturbed by up to half a
    decade per component reaches them (1e-8 in log10) on every sample;
  - from the reference's cold start (each component's species at its total)
    Newton converges on a quarter of the samples in 200 iterations (the
    reference's PCF + Anderson on 58 of 64): where it does, it reaches the
    known answer and the species of the reference's converged PCF solves to
    1e-6 relative.
"""
import os

import numpy as np
import pytest

from oracle import oracle as o

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "uranium_tableau.npz")


@pytest.fixture(scope="module")
def ur(pkg):
    d = np.load(GOLD)
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, d["S"], d["logk"], list(d["comp_species"]), max_iter=200, tol=1e-10, warm_iter=8,
                      anderson_depth=4)
    return d, sys_


def test_tableau_shape(ur):
    d, sys_ = ur
    assert d["S"].shape == (95, 17) and sys_.n_comp == 17 and sys_.n_species == 95
    assert (d["comp_species"] >= 0).all()


@pytest.mark.parametrize("start", ["cstar", "cold"])
def test_oracle_pcf_reproduces_reference_solver(ur, start):
    d, sys_ = ur
    species = d["cstar"] if start == "cstar" else d["cold"]
    out, it, cv = o.pcf_batch(sys_, species)
    key = "pcf" if start == "cstar" else "pcf_cold"
    np.testing.assert_array_equal(cv, d[key + "_cv"])
    np.testing.assert_array_equal(it, d[key + "_it"])
    np.testing.assert_allclose(out, d[key + "_out"], rtol=1e-12, atol=1e-300)


def test_oracle_newton_reaches_known_answers_from_near(ur, pkg):
    d, _ = ur
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, d["S"], d["logk"], list(d["comp_species"]), max_iter=200, tol=1e-10, warm_iter=50)
    rng = np.random.default_rng(1)
    x0 = d["xstar"] + rng.uniform(-0.5, 0.5, d["xstar"].shape)
    x, it, st = o.eq_batch(sys_, d["totals"], d["cold"], x0=x0, start=1)
    assert (st == 0).all(), (st, it)
    assert np.abs(x - d["xstar"]).max() <= 1e-8
    assert it.max() <= 20


def test_oracle_newton_from_cold_start(ur):
    d, sys_ = ur
    x, it, st = o.eq_batch(sys_, d["totals"], d["cold"], start=0)
    ok = st <= 1
    assert ok.mean() >= 0.2, (ok.mean(), it)
    assert np.abs(x[ok] - d["xstar"][ok]).max() <= 1e-8
    # the species of the reference's converged PCF solves from the same cold vectors
    c = np.zeros((x.shape[0], 95))
    for k in range(x.shape[0]):
        cc = np.zeros(95)
        o.lib().orc_eq_species(__import__("ctypes").byref(sys_), o._p(np.ascontiguousarray(x[k])), o._p(cc))
        c[k] = cc
    both = ok & (d["pcf_cold_cv"] == 1)
    active = np.abs(d["S"]).sum(1) > 0
    ref = d["pcf_cold_out"][both][:, active]
    got = c[both][:, active]
    big = ref > 1e-25
    assert np.max(np.abs(got[big] - ref[big]) / ref[big]) <= 1e-6
