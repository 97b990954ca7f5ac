"""The oracle's restatement of the reference's live speciation solver (PCF +
Anderson acceleration, calculate_species_concentrations) on the CPU: against
the golden fixtures made from the reference's own code, and against that code
compiled from its sources (oracle/_ref) on fresh inputs, including starts the
solver does not converge from.  Same compiler, same operation order: the
iteration counts, convergence flags and species agree exactly."""
import os

import numpy as np
import pytest

from oracle import oracle as o

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _sys(pkg, S, logk, cs, max_iter=200, tol=1e-10, depth=4):
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, list(cs), max_iter=max_iter, tol=tol, solver=pkg.EQ_SOLVER_PCF,
                      anderson_depth=depth)
    return sys_


def test_pcf_carbonate_fixture(pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    out, it, cv = o.pcf_batch(_sys(pkg, z["S4"], z["logk4"], [0, 1]), z["species4"])
    np.testing.assert_array_equal(it, z["it4"])
    np.testing.assert_array_equal(cv, z["cv4"])
    np.testing.assert_array_equal(out, z["out4"])


def test_pcf_random_tableau_fixture(pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    out, it, cv = o.pcf_batch(_sys(pkg, z["S"], z["logk"], z["comp_species"]), z["cstar"])
    np.testing.assert_array_equal(it, z["pcf_it"])
    np.testing.assert_array_equal(cv, z["pcf_cv"])
    np.testing.assert_array_equal(out, z["pcf_out"])


def _hard_inputs(S, n, seed):
    """Every species drawn log-uniform over 1e-6..1: the solver takes a
    hundred iterations on the median input and does not converge in 200 on
    about a quarter of them."""
    rng = np.random.default_rng(seed)
    return 10.0 ** rng.uniform(-6, 0, size=(n, S.shape[0]))


@pytest.mark.parametrize("depth,max_iter", [(4, 200), (2, 60), (1, 30)])
def test_pcf_matches_reference_code(pkg, depth, max_iter):
    if o.ref_lib() is None:
        pytest.skip("reference tree absent: oracle/_ref not built")
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    S, logk = z["S"], z["logk"]
    cs = list(range(S.shape[1]))
    c = _hard_inputs(S, 300, seed=depth)
    out, it, cv = o.pcf_batch(_sys(pkg, S, logk, cs, max_iter=max_iter, depth=depth), c)
    rout, rit, rcv = o.ref_pcf_solve(S, logk, cs, c, max_iter=max_iter, tol=1e-10, depth=depth)
    assert 0 < cv.sum() < cv.size          # both outcomes are exercised
    np.testing.assert_array_equal(it, rit)
    np.testing.assert_array_equal(cv, rcv)
    np.testing.assert_array_equal(out, rout)
