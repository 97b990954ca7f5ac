"""Fused multi-solute D3Q7 transport + reaction step on the GPU against the FP64 oracle.

Tolerances (FP32 populations vs FP64 oracle):
  solute concentration fields: relative L2 <= 1e-5 (transport only) and
  <= 1e-4 with reactions; biomass (FP64 field, FP32-driven rates) <= 1e-5.
  Mask updates (integer): bit-exact.
"""
import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def flow_field(pkg, cfg, mask, steps=400):
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(steps)
    lat.couple_velocity()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, k).reshape(-1) for k in range(3)])
    return lat, u


@pytest.mark.parametrize("steps", [1, 2, 5, 120])
def test_single_solute_breakthrough(gpu_lib, pkg, wl, steps):
    """One solute, C=1 Dirichlet inlet, zero-gradient outlet, C=0 initially,
    velocity from the flow lattice (the 64^3 case's transport, reduced)."""
    mask = wl.sphere_pack(22, 16, 16, 0.5, 2.0, 4.0, seed=5)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0,
                          solutes=[{"tau": 0.7, "c0": 0.0, "left": "D", "left_value": 1.0, "right": "N"}])
    lat, u = flow_field(pkg, cfg, mask)
    lat.ade_init()
    lat.step(steps)
    ref = o.Transport(cfg, mask, u=u)
    ref.step(steps)
    cg = lat.field(pkg.FIELD_CONC, 0).reshape(-1)
    co = ref.density(0)
    assert rel_l2(cg, co) < 1e-5
    # outlet breakthrough (mean C at x = nx-2)
    bg = cg.reshape(nx, ny, nz)[nx - 2].mean()
    bo = co.reshape(nx, ny, nz)[nx - 2].mean()
    assert bg == pytest.approx(bo, rel=1e-4, abs=1e-7)
    lat.close()


def test_closed_mass_conservation(gpu_lib, pkg, wl):
    mask = wl.sphere_pack(24, 12, 12, 0.6, 2, 3, seed=1)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.9}, {"tau": 0.6}])
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    rng = np.random.default_rng(0)
    c = np.zeros((nx, ny, nz)); c[9:15] = rng.uniform(0, 1, (6, ny, nz))
    lat.set_field(pkg.FIELD_CONC, 0, c)
    lat.set_field(pkg.FIELD_CONC, 1, 2 * c)
    m0 = [lat.reduce(pkg.FIELD_CONC, s, pkg.RED_SUM) for s in range(2)]
    lat.step(5)
    for s in range(2):
        assert lat.reduce(pkg.FIELD_CONC, s, pkg.RED_SUM) == pytest.approx(m0[s], rel=2e-6)
    lat.close()


def _biotic_cfg(pkg, wl, nx, ny, nz, seed=2):
    rng = np.random.default_rng(seed)
    taus = rng.uniform(0.6, 0.9, 4)
    sol = [{"tau": float(taus[0]), "c0": 0.05, "left": "D", "left_value": 0.1, "right": "N"},
           {"tau": float(taus[1]), "c0": 0.02, "left": "D", "left_value": 0.05, "right": "N"},
           {"tau": float(taus[2]), "c0": 0.03, "left": "D", "left_value": 0.03, "right": "N"},
           {"tau": float(taus[3]), "c0": 0.0, "left": "D", "left_value": 0.0, "right": "N"}]
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0, solutes=sol, microbes=1, dt=50.0)
    cfg.enable_kinetics = 1
    vmax = rng.uniform(1e-5, 1e-4, 2); ks = rng.uniform(1e-3, 1e-1, 3)
    # dual Monod on the donor (0) with O2 (1) or NO3- (2); product (3)
    pkg.add_rxn(cfg, microbe=0, k=float(vmax[0]), monod=[(0, float(ks[0])), (1, float(ks[1]))],
                nu={0: -1.0, 1: -0.5, 3: 1.0}, yield_=0.3)
    pkg.add_rxn(cfg, microbe=0, k=float(vmax[1]), monod=[(0, float(ks[0])), (2, float(ks[2]))],
                nu={0: -1.0, 2: -0.8, 3: 1.0}, yield_=0.2)
    cfg.decay[0] = 1e-6
    return cfg


def _seed_biomass(mask, seed, frac=0.02):
    rng = np.random.default_rng(seed)
    pore = mask == 2
    near = np.zeros_like(pore)
    solid = (mask == 0) | (mask == 1)
    for ax in range(3):
        for sh in (1, -1):
            near |= np.roll(solid, sh, axis=ax)
    cand = np.argwhere(pore & near)
    pick = cand[rng.random(len(cand)) < frac * 5]
    b = np.zeros(mask.shape)
    b[tuple(pick.T)] = rng.uniform(10, 50, len(pick))
    b[0] = 0; b[-1] = 0
    return b


def test_biotic_dual_monod(gpu_lib, pkg, wl):
    mask = wl.sphere_pack(26, 16, 16, 0.5, 2.0, 4.0, seed=9)
    nx, ny, nz = mask.shape
    cfg = _biotic_cfg(pkg, wl, nx, ny, nz)
    lat, u = flow_field(pkg, cfg, mask)
    lat.ade_init()
    b = _seed_biomass(mask, 4)
    lat.set_field(pkg.FIELD_BIOMASS, 0, b)
    ref = o.Transport(cfg, mask, u=u)
    ref.set_biomass(0, b)
    for n in (1, 3, 30):
        lat.step(n)
        ref.step(n)
    for s in range(4):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    assert rel_l2(lat.field(pkg.FIELD_BIOMASS, 0).reshape(-1), ref.biomass(0)) < 1e-5
    lat.close()


def test_precipitation_surface_and_mask(gpu_lib, pkg, wl):
    """Example-13 chemistry: Fe + HS -> FeS(s) on wall-adjacent voxels, FeS
    immobile; then node conversion, bit-exact on identical inventories."""
    mask = wl.sphere_pack(20, 14, 14, 0.55, 2.0, 3.0, seed=13)
    nx, ny, nz = mask.shape
    sol = [{"tau": 0.8, "c0": 0.5, "left": "D", "left_value": 5.0, "right": "N"},
           {"tau": 0.8, "c0": 0.5, "left": "N", "right": "D", "right_value": 5.0},
           {"immobile": True, "c0": 0.0}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, dt=0.01)
    cfg.enable_abiotic = 1
    cfg.precip_enabled = 1
    cfg.abiotic_surface_only = 1
    cfg.precip_substrate = 2
    cfg.max_precip_rho = 0.8      # about the median inventory after 60 steps
    cfg.precip_code = 0
    pkg.add_rxn(cfg, k=20.0, mass=[0, 1], nu={0: -1.0, 1: -1.0, 2: 1.0})
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    ref = o.Transport(cfg, mask)
    lat.step(60)
    ref.step(60)
    for s in range(3):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    # conversion kernel bit-exact given the same inventory
    inv = ref.density(2)
    lat.set_field(pkg.FIELD_CONC, 2, inv)
    ch_g = lat.precip_convert()
    ch_o = ref.precip_convert()
    assert ch_g == ch_o and 0 < ch_o < int((inv > 0).sum())
    np.testing.assert_array_equal(lat.mask().reshape(-1), ref.mask)
    assert lat.reduce(pkg.FIELD_CONC, 0, pkg.RED_COUNT_EQ, 0) == float((ref.mask == 0).sum())
    lat.close()


def test_equilibrium_in_transport_carbonate(gpu_lib, pkg, wl):
    """Example 04's carbonate tableau as the transported solutes, Newton each step."""
    mask = wl.sphere_pack(16, 10, 10, 0.6, 2.0, 3.0, seed=21)
    nx, ny, nz = mask.shape
    sol = [{"tau": 0.8, "c0": 1e-3, "left": "D", "left_value": 2e-3, "right": "N"},
           {"tau": 0.8, "c0": 1e-7, "left": "D", "left_value": 1e-6, "right": "N"},
           {"tau": 0.8, "c0": 1e-30, "left": "D", "left_value": 1e-30, "right": "N"},
           {"tau": 0.8, "c0": 1e-30, "left": "D", "left_value": 1e-30, "right": "N"}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol)
    cfg.use_equilibrium = 1
    S = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], float)
    pkg.set_eq_system(cfg.eq, S, [0.0, 0.0, -10.33, 6.35], [0, 1], max_iter=100, tol=1e-10)
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
        assert rel_l2(cg, co) < 1e-4, s
    lat.close()


def test_coupled_warm_previous_matches_cold(gpu_lib, pkg, wl):
    """The coupled chemistry with Newton started from each voxel's previous
    solution gives the same fields as the reference's cold start (both stop
    at the 1e-10 relative residual) and needs fewer iterations."""
    mask = wl.sphere_pack(24, 16, 16, 0.5, 2.0, 4.0, seed=17)
    nx, ny, nz = mask.shape
    bio = wl.seed_biomass(mask, 3, frac=0.2)
    out = {}
    for warm in (False, True):
        cfg = wl.coupled_config(pkg, nx, ny, nz, warm_previous=warm)
        lat = pkg.Lattice(cfg)
        lat.upload_mask(mask)
        lat.flow_init()
        lat.flow_steps(50)
        lat.couple_velocity()
        lat.ade_init()
        lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
        st = lat.step(30)
        assert st == pkg.OK
        it = lat.field(pkg.FIELD_EQ_ITERS).reshape(-1)[(mask == 2).reshape(-1)]
        out[warm] = ([lat.field(pkg.FIELD_CONC, s).reshape(-1) for s in range(cfg.n_solutes)], it.mean())
        lat.close()
    for s in range(len(out[False][0])):
        assert rel_l2(out[True][0][s], out[False][0][s]) < 1e-6, s
    assert out[True][1] < out[False][1]


def test_surrogate_reaction_type(gpu_lib, pkg, wl):
    """Two surrogate organisms (3->20->20->4 networks) on sessile biomass feed
    six transported solutes; the fused step against the FP64 oracle (the
    network runs in FP32 on the GPU)."""
    mask = wl.sphere_pack(22, 14, 14, 0.5, 2.0, 3.0, seed=23)
    nx, ny, nz = mask.shape
    cfg = wl.surrogate_config(pkg, nx, ny, nz)
    nets = wl.surrogate_nets(pkg)
    rng = np.random.default_rng(8)
    b0 = wl.seed_biomass(mask, 4, frac=0.3, lo=0.005, hi=0.05)
    b1 = wl.seed_biomass(mask, 5, frac=0.3, lo=0.005, hi=0.05)
    lat, u = flow_field(pkg, cfg, mask, steps=100)
    for slot in range(2):
        lat.set_surrogate(slot, nets[slot])
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, b0)
    lat.set_field(pkg.FIELD_BIOMASS, 1, b1)
    ref = o.Transport(cfg, mask, u=u)
    ref.set_surrogates(nets)
    ref.set_biomass(0, b0)
    ref.set_biomass(1, b1)
    for n in (1, 4, 20):
        lat.step(n)
        ref.step(n)
    for s in range(6):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    for m in range(2):
        bg, bo = lat.field(pkg.FIELD_BIOMASS, m).reshape(-1), ref.biomass(m)
        assert rel_l2(bg, bo) < 1e-5, m
        assert not np.allclose(bo, (b0, b1)[m].reshape(-1))      # the organisms did something
    lat.close()


def test_set_transport_ignores_immobile_relaxation(gpu_lib, pkg, wl):
    """The driver derives every solute's relaxation from its diffusion
    coefficient; an immobile solute (D = 0) gets 2, outside (0, 2), and has
    no lattice to relax: accepted and ignored.  A mobile one at 2 is refused."""
    mask = wl.sphere_pack(12, 8, 8, 0.6, 1.5, 2.5, seed=3)
    cfg = pkg.make_config(*mask.shape, solutes=[{"tau": 0.8}, {"immobile": True}])
    lat = pkg.Lattice(cfg)
    lat.set_transport([1.25, 2.0], [1.25, 2.0], 0.01)
    with pytest.raises(pkg.CLError):
        lat.set_transport([2.0, 2.0], [2.0, 2.0], 0.01)
    lat.close()


def test_lbm_solved_microbe_carried_by_a_solute(gpu_lib, pkg, wl):
    """A microbe solved by LBM (the reference's planktonic bFree lattice):
    solute 2 carries its biomass, advected and diffused with its own
    relaxation; dual-Monod growth on solutes 0 and 1 reads that density and
    adds to it.  Against the oracle after 1, 4 and 34 steps (rel. L2 <= 1e-4);
    the sessile field stays zero."""
    mask = wl.sphere_pack(26, 16, 16, 0.5, 2.0, 4.0, seed=19)
    nx, ny, nz = mask.shape
    sol = [{"tau": 0.8, "c0": 0.05, "left": "D", "left_value": 0.2, "right": "N"},
           {"tau": 0.7, "c0": 0.02, "left": "D", "left_value": 0.1, "right": "N"},
           {"tau": 0.55, "c0": 1.0, "left": "N", "right": "N"}]
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.0005, rho_out=1.0, solutes=sol, microbes=1, dt=1.0)
    cfg.enable_kinetics = 1
    pkg.add_rxn(cfg, microbe=0, k=2e-3, monod=[(0, 5e-2), (1, 1e-2)], nu={0: -1.0, 1: -0.5}, yield_=0.4)
    cfg.decay[0] = 1e-5
    cfg.microbe_carrier[0] = 3
    lat, u = flow_field(pkg, cfg, mask)
    lat.ade_init()
    ref = o.Transport(cfg, mask, u=u)
    for n in (1, 3, 30):
        lat.step(n)
        ref.step(n)
        for s in range(3):
            assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, (n, s)
    assert not np.allclose(ref.density(2), ref.density(2)[0])      # the biomass grew unevenly
    assert np.all(lat.field(pkg.FIELD_BIOMASS, 0) == 0.0)
    lat.close()
