"""Pin the FP64 oracle before trusting it (CPU only).

- known answers of the reference's own code compiled from its sources
  (oracle/_ref): example 04's carbonate tableau and the shipped surrogate;
- the oracle's Newton against the reference's PCF + Anderson solver on
  samples where both converge;
- the oracle's table-driven rate law against the example rate-law headers;
- the oracle's MLP gradients against finite differences;
- LBM restatement against analytic solutions (Poiseuille, linear diffusion).
"""
import numpy as np
import pytest

from oracle import oracle as o

CARBONATE_S = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], float)
CARBONATE_LOGK = np.array([0.0, 0.0, -10.33, 6.35])


def need_ref():
    if o.ref_lib() is None:
        pytest.skip("reference tree not present: oracle/_ref not built")


def test_ref_carbonate_known_answer():
    need_ref()
    out, it, cv = o.ref_pcf_solve(CARBONATE_S, CARBONATE_LOGK, [0, 1], [1e-3, 1e-7, 1e-30, 1e-30])
    want = [9.799444e-4, 4.592678e-9, 9.980112e-6, 1.007552e-5]
    assert cv[0] == 1 and it[0] == 7
    np.testing.assert_allclose(out[0], want, rtol=1e-6)


def test_ref_surrogate_known_answer():
    need_ref()
    assert o.ref_surrogate([5.0, 0.2])[0] == pytest.approx(2.2985048920885152e-07, rel=1e-14)


def _eq_sys(pkg, S, logk, cs, **kw):
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, cs, **kw)
    return sys_


def test_oracle_newton_carbonate(pkg):
    need_ref()
    sys_ = _eq_sys(pkg, CARBONATE_S, CARBONATE_LOGK, [0, 1], max_iter=100, tol=1e-12)
    sp = np.array([[1e-3, 1e-7, 1e-30, 1e-30]])
    T = np.zeros((1, 2))
    T[0] = np.maximum(np.clip(sp[0], 1e-30, 10) @ CARBONATE_S, 1e-30)
    x, it, st = o.eq_batch(sys_, T, sp, start=0)
    assert st[0] == 0
    c = 10 ** (CARBONATE_LOGK + CARBONATE_S @ x[0])
    ref, _, _ = o.ref_pcf_solve(CARBONATE_S, CARBONATE_LOGK, [0, 1], sp[0])
    np.testing.assert_allclose(c, ref[0], rtol=1e-6)


def test_oracle_newton_vs_reference_pcf(pkg, wl):
    """5 components x 14 species: both solvers on the same well-posed totals;
    where the reference converged without a clamp, the species agree."""
    need_ref()
    S, logk, cs = wl.tableau(5, 9, seed=4)
    T, xs, cstar, acc = wl.speciation_batch(S, logk, 300, seed=11)
    sys_ = _eq_sys(pkg, S, logk, cs, max_iter=200, tol=1e-10)
    x, it, st = o.eq_batch(sys_, T, wl.cold_species(S, T, cs), start=0)
    conv = st == 0
    assert conv.mean() > 0.9
    # Newton recovers the planted free concentrations
    np.testing.assert_allclose(x[conv], xs[conv], atol=1e-7)
    # the reference PCF+AA from the species it would hold at equilibrium
    ref, rit, rcv = o.ref_pcf_solve(S, logk, cs, cstar)
    both = conv & (rcv == 1)
    assert both.sum() > 50
    c_newton = 10 ** (logk[None, :] + x @ S.T)
    rel = np.abs(ref[both] - c_newton[both]) / np.maximum(c_newton[both], 1e-300)
    big = c_newton[both] > 1e-25
    assert np.median(rel[big]) < 1e-6


def test_oracle_rates_match_example_headers(pkg):
    need_ref()
    # examples/05: Monod growth on C[0], product C[1], two microbes
    cfg = pkg.make_config(5, 4, 4, solutes=[{}, {}], microbes=2)
    mu, Ks, Y, fP, kd = [2e-4, 1e-4], [5e-2, 5e-3], [0.4, 0.4], [2.0, 2.0], [1e-6, 1e-6]
    for m in range(2):
        pkg.add_rxn(cfg, microbe=m, k=mu[m], monod=[(0, Ks[m])], nu={0: -1.0 / Y[m], 1: fP[m]}, yield_=1.0)
        cfg.decay[m] = kd[m]
    rng = np.random.default_rng(5)
    for _ in range(50):
        C = rng.uniform(0, 0.2, 2); B = rng.uniform(0, 50, 2)
        R, BR = o.rates(cfg, 0, C, B)
        rR, rBR = o.ref_kinetics_ex05(B, C)
        np.testing.assert_allclose(R, rR, rtol=1e-13, atol=1e-300)
        np.testing.assert_allclose(BR, rBR, rtol=1e-13, atol=1e-300)
    # examples/13: R = k Fe HS, Fe + HS -> FeS
    cfg = pkg.make_config(5, 4, 4, solutes=[{}, {}, {"immobile": True}])
    pkg.add_rxn(cfg, k=20.0, mass=[0, 1], nu={0: -1.0, 1: -1.0, 2: 1.0})
    for _ in range(50):
        C = rng.uniform(0, 5, 3)
        R, _ = o.rates(cfg, 1, C)
        np.testing.assert_allclose(R, o.ref_abiotic_ex13(C), rtol=1e-13)


def test_oracle_mlp_gradient_finite_difference():
    rng = np.random.default_rng(0)
    n_in, H, n_out = 5, 8, 5
    npar = H * n_in + H + H * H + H + n_out * H + n_out
    p = rng.normal(0, 0.5, npar)
    x = rng.normal(0, 1, (7, n_in)); y = rng.normal(0, 1, (7, n_out))
    loss, g, _ = o.mlp_forward_backward(n_in, H, n_out, p, x, y)
    eps = 1e-6
    for k in rng.choice(npar, 25, replace=False):
        pp = p.copy(); pp[k] += eps
        lp, _, _ = o.mlp_forward_backward(n_in, H, n_out, pp, x, y, want_grad=False)
        pm = p.copy(); pm[k] -= eps
        lm, _, _ = o.mlp_forward_backward(n_in, H, n_out, pm, x, y, want_grad=False)
        assert g[k] == pytest.approx((lp - lm) / (2 * eps), rel=1e-5, abs=1e-9)


def test_oracle_poiseuille(pkg, wl):
    """Pressure-driven plane channel: parabolic profile, walls half-way to the
    bounce-back nodes."""
    nx, ny, nz = 24, 18, 3
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.0005, rho_out=1.0)
    fl = o.Flow(cfg, wl.channel(nx, ny, nz))
    it, _ = fl.solve(20000, 1e-9)
    assert 500 <= it < 20000
    rho, u = fl.macro()
    ux = u[0].reshape(nx, ny, nz)[nx // 2, :, 1]
    nu = (0.8 - 0.5) / 3.0
    G = (1.0 / 3.0) * (cfg.rho_in - cfg.rho_out) / (nx - 1)
    y = np.arange(ny)
    ana = G / (2 * nu) * (y - 0.5) * (ny - 1.5 - y)
    ana[0] = ana[-1] = 0.0
    err = np.linalg.norm(ux[1:-1] - ana[1:-1]) / np.linalg.norm(ana[1:-1])
    assert err < 0.02, err


def test_oracle_linear_diffusion_profile(pkg):
    """Example 02's known answer: steady diffusion between Dirichlet 1 and 0 is
    a straight line."""
    nx, ny, nz = 18, 2, 2
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 1.0, "c0": 0.0, "left": "D", "left_value": 1.0,
                                                "right": "D", "right_value": 0.0}])
    mask = np.full((nx, ny, nz), 2, np.uint8)
    tr = o.Transport(cfg, mask)
    tr.step(6000)
    c = tr.density(0).reshape(nx, ny, nz)[:, 0, 0]
    # Dirichlet density holds at the boundary nodes; linear in between
    lin = np.polyfit(np.arange(nx), c, 1)
    assert np.max(np.abs(np.polyval(lin, np.arange(nx)) - c)) < 1e-6
    assert c[0] == pytest.approx(1.0, abs=1e-9) and c[-1] == pytest.approx(0.0, abs=1e-9)


def test_oracle_transport_conserves_mass_closed(pkg, wl):
    """Zero-gradient faces, no flow, no reaction: total solute is conserved up
    to the boundary planes' exchange; interior diffusion alone is exact."""
    nx, ny, nz = 20, 10, 10
    mask = wl.sphere_pack(nx, ny, nz, 0.6, 2, 3, seed=1)
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.9, "c0": 0.0}])
    tr = o.Transport(cfg, mask)
    rng = np.random.default_rng(0)
    c = np.zeros((nx, ny, nz)); c[8:12] = rng.uniform(0, 1, (4, ny, nz))
    tr.set_conc(0, c)
    m0 = tr.density(0).sum()
    tr.step(4)
    assert tr.density(0).sum() == pytest.approx(m0, rel=1e-12)
