"""The reference's live speciation solver (PCF + Anderson acceleration) on the
GPU: the batch entry point cl_eq_pcf_host against the golden fixtures made from
the reference's own code and against the oracle's restatement (which matches
that code exactly), and the transport step with eq.solver = PCF against the
oracle stepped the same way.

Tolerances.  The device rounds sums and products one operation at a time as
the reference does, but its exp10 / log10 are CUDA's, so an iterate can differ
in the last bits:
  - the golden fixtures (well-posed inputs): convergence flags equal on
    >= 95 %, iteration counts equal on >= 90 % and within 3 on the converged
    solves, species to rel 1e-9 (a solve that stops at ||f||_2 < 1e-10, f a
    log10 ratio, fixes them to about ln(10) * 1e-10 there);
  - random inputs on which the iteration wanders for tens to hundreds of
    steps: the reference's own outcome there depends on the last bits of its
    input, so the GPU is held to the oracle's disagreement with itself on
    inputs scaled by 1 + 2^-50 (flags, iterations within 3, converged species);
  - the transport step: relative L2 <= 1e-4, the bar of the other transport
    tests (FP32 populations against FP64).
"""
import os

import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "tests", "golden")


def _sys(pkg, S, logk, cs, max_iter=200, tol=1e-10, depth=4):
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, list(cs), max_iter=max_iter, tol=tol, solver=pkg.EQ_SOLVER_PCF,
                      anderson_depth=depth)
    return sys_


def _compare(out, it, cv, rout, rit, rcv):
    """Well-posed inputs: the same flags and (nearly) the same iterations."""
    both = (cv == 1) & (rcv == 1)
    np.testing.assert_allclose(out[both], rout[both], rtol=1e-9, atol=1e-30)
    assert (cv == rcv).mean() >= 0.95
    assert (it == rit).mean() >= 0.90
    assert np.abs(it[both].astype(int) - rit[both]).max() <= 3


def _compare_vs_perturbed(out, it, cv, sys_, c):
    """Inputs the iteration wanders on: there an ulp of exp10 / log10 changes
    the trajectory, and the reference's own outcome changes with the last bits
    of its input.  The yardstick is the oracle (which matches the reference
    exactly) against itself on the inputs scaled by 1 + 2^-50: the GPU may
    differ from the oracle about as much, and no more.  ||f||_2 < tol bounds
    the log-ratio of each component's balance, not the free concentrations,
    so two converged solves of an ill-conditioned tableau can sit ~1e-7
    apart; the same yardstick sets that bar."""
    rout, rit, rcv = o.pcf_batch(sys_, c)
    pout, pit, pcv = o.pcf_batch(sys_, c * (1.0 + 2.0 ** -50))
    assert (cv != rcv).mean() <= (pcv != rcv).mean() + 0.03
    assert (np.abs(it.astype(int) - rit) <= 3).mean() >= (np.abs(pit.astype(int) - rit) <= 3).mean() - 0.05
    both, pboth = (cv == 1) & (rcv == 1), (pcv == 1) & (rcv == 1)
    rel = np.abs(out[both] - rout[both]) / rout[both]
    prel = np.abs(pout[pboth] - rout[pboth]) / rout[pboth]
    assert rel.max() <= 1e-5
    assert np.quantile(rel, 0.999) <= max(10 * np.quantile(prel, 0.999), 1e-9)
    assert np.median(rel) <= max(10 * np.median(prel), 1e-10)
    return rcv


def test_pcf_batch_golden_carbonate(gpu_lib, pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    s = pkg.EqSolver(_sys(pkg, z["S4"], z["logk4"], [0, 1]))
    out, it, cv = s.pcf(z["species4"])
    np.testing.assert_array_equal(cv, z["cv4"])
    assert np.abs(it - z["it4"]).max() <= 1
    np.testing.assert_allclose(out, z["out4"], rtol=1e-9, atol=1e-30)
    s.close()


def test_pcf_batch_golden_random_tableau(gpu_lib, pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    s = pkg.EqSolver(_sys(pkg, z["S"], z["logk"], z["comp_species"]))
    out, it, cv = s.pcf(z["cstar"])
    _compare(out, it, cv, z["pcf_out"], z["pcf_it"], z["pcf_cv"])
    s.close()


@pytest.mark.parametrize("depth,max_iter", [(4, 200), (1, 50), (8, 200)])
def test_pcf_batch_matches_oracle(gpu_lib, pkg, depth, max_iter):
    """Every species log-uniform over 1e-6..1 on the 5 x 14 tableau: the solver
    needs about a hundred iterations on the median input and fails on about a
    quarter, so both outcomes and the whole Anderson path are exercised."""
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    S, logk = z["S"], z["logk"]
    sys_ = _sys(pkg, S, logk, range(5), max_iter=max_iter, depth=depth)
    c = 10.0 ** np.random.default_rng(depth).uniform(-6, 0, size=(4000, 14))
    s = pkg.EqSolver(sys_)
    out, it, cv = s.pcf(c)
    rcv = _compare_vs_perturbed(out, it, cv, sys_, c)
    assert 0 < rcv.sum() < rcv.size
    s.close()


@pytest.mark.parametrize("nc", [1, 2, 3])
def test_pcf_batch_component_counts(gpu_lib, pkg, nc):
    """Sub-tableaux of 1..3 components (the instantiations the transport step
    uses for small systems)."""
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    S = z["S"][:, :nc]
    keep = np.abs(S).sum(1) > 0
    S, logk = S[keep], z["logk"][keep]
    sys_ = _sys(pkg, S, logk, range(nc))
    c = 10.0 ** np.random.default_rng(nc).uniform(-6, -1, size=(2000, S.shape[0]))
    s = pkg.EqSolver(sys_)
    out, it, cv = s.pcf(c)
    _compare_vs_perturbed(out, it, cv, sys_, c)
    s.close()


def test_pcf_rejects_depth(gpu_lib, pkg):
    z = np.load(os.path.join(GOLD, "speciation_pcf.npz"))
    with pytest.raises(pkg.CLError):
        pkg.EqSolver(_sys(pkg, z["S4"], z["logk4"], [0, 1], depth=9))


def test_pcf_in_transport_carbonate(gpu_lib, pkg, wl):
    """Example 04's carbonate tableau as the transported solutes with the
    reference's live solver every step: the GPU against the oracle stepped the
    same way, and the iteration counts of the last step."""
    mask = wl.sphere_pack(16, 10, 10, 0.6, 2.0, 3.0, seed=21)
    nx, ny, nz = mask.shape
    sol = [{"tau": 0.8, "c0": 1e-3, "left": "D", "left_value": 2e-3, "right": "N"},
           {"tau": 0.8, "c0": 1e-7, "left": "D", "left_value": 1e-6, "right": "N"},
           {"tau": 0.8, "c0": 1e-30, "left": "D", "left_value": 1e-30, "right": "N"},
           {"tau": 0.8, "c0": 1e-30, "left": "D", "left_value": 1e-30, "right": "N"}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol)
    cfg.use_equilibrium = 1
    S = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], float)
    pkg.set_eq_system(cfg.eq, S, [0.0, 0.0, -10.33, 6.35], [0, 1], max_iter=200, tol=1e-10,
                      solver=pkg.EQ_SOLVER_PCF)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    ref = o.Transport(cfg, mask)
    st = lat.step(25)
    nc = ref.step(25)
    assert nc == 0 and st == pkg.OK
    for s in range(4):
        cg = lat.field(pkg.FIELD_CONC, s).reshape(-1)
        co = ref.density(s)
        assert np.linalg.norm(cg - co) <= 1e-4 * np.linalg.norm(co), s
    pore = (mask.reshape(-1) == 2)
    it_g = lat.field(pkg.FIELD_EQ_ITERS).reshape(-1)[pore]
    it_o = ref.eq_iters[pore]
    assert it_g.mean() > 1 and abs(it_g.mean() - it_o.mean()) <= 0.1 * it_o.mean()
    lat.close()


def test_pcf_in_coupled_chemistry(gpu_lib, pkg, wl):
    """The coupled workload's 3-component chemistry (kinetics, surface
    precipitation, speciation) with the live solver.  A few voxels per step
    do not converge in 200 iterations and the reference applies whatever the
    solve ended at, which depends chaotically on the input: perturbing the
    oracle's starting concentrations by 1e-7 (FP32 storage) moves the
    equilibrium species by ~1e-3 after 12 steps, where Newton (which applies
    nothing unconverged) moves them by ~1e-7.  Bars: the solutes outside the
    speciation to the transport tolerance 1e-4, the equilibrium species to
    three times the oracle's own spread under that perturbation."""
    mask = wl.sphere_pack(20, 12, 12, 0.5, 2.0, 3.0, seed=23)
    nx, ny, nz = mask.shape
    cfg = wl.coupled_config(pkg, nx, ny, nz, warm_previous=False)
    cfg.eq.solver = pkg.EQ_SOLVER_PCF
    cfg.eq.max_iter = 200
    bio = wl.seed_biomass(mask, 3, frac=0.2)
    steps = 12
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
    lat.step(steps)
    ref, pert = o.Transport(cfg, mask), o.Transport(cfg, mask)
    rng = np.random.default_rng(1)
    for t in (ref, pert):
        t.set_biomass(0, bio)
    for s in range(8):
        c = pert.density(s)
        pert.set_conc(s, c * (1 + 1e-7 * rng.standard_normal(c.size)))
    ref.step(steps)
    pert.step(steps)
    eq_species = [s for s in range(cfg.n_solutes) if np.abs(np.asarray(cfg.eq.stoich[s])[:3]).sum() > 0]
    for s in range(cfg.n_solutes):
        cg, co = lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)
        spread = np.linalg.norm(pert.density(s) - co)
        bar = 1e-4 * np.linalg.norm(co) + 1e-25
        if s in eq_species:
            bar = max(bar, 3 * spread)
        assert np.linalg.norm(cg - co) <= bar, s
    lat.close()
