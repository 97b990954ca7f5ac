"""The oracle's reaction stage and node conversions against the reference's own
processors (CPU): run_kinetics, update_rxnLattices, surfaceAbioticKinetics3D /
run_abiotic_kinetics, surfaceDissolutionKinetics3D, update_abiotic_rxnLattices,
run_equilibrium_biotic, precipNodeConversion3D and dissolNodeConversion3D,
compiled from the reference's sources with the rate laws of examples 05, 13
and 14 (oracle/ref/rxn_harness.cpp) and run on one block.

Tolerances: the reference keeps every scalar as seven populations offset by
the lattice weights (the density is 1 + their sum), so each value it stores
or increments carries an absolute rounding of ~1e-16; concentrations agree
to rel 1e-10 + abs 1e-14, biomass (O(10)) to rel 1e-12.  The equilibrium
step solves with the reference's PCF + Anderson there and, in the oracle,
Newton (both to a 1e-10 residual: rel 1e-6) or the restated PCF + Anderson
(rel 5e-10 + abs 1e-14).  Masks and phases: bit-exact.
"""
import numpy as np
import pytest

from oracle import oracle as o

FULL = 27.1


def need(variant):
    if o.rxn_lib(variant) is None:
        pytest.skip("reference tree absent: oracle/_ref not built")


def geometry(nx, ny, nz, seed, grain_code=0):
    rng = np.random.default_rng(seed)
    mask = np.full((nx, ny, nz), 2, np.uint8)
    for _ in range(8):
        x, y, z = rng.integers(1, nx - 3), rng.integers(1, ny - 3), rng.integers(0, nz - 2)
        mask[x:x + 2, y:y + 2, z:z + 2] = grain_code
    # walls on the four y / z faces: the oracle's surface gate and dissolution
    # faces wrap y and z with the periodic transport, the reference's stop at
    # the domain edge; with walls there the two read the same neighbours
    mask[:, 0, :] = mask[:, ny - 1, :] = 1
    mask[:, :, 0] = mask[:, :, nz - 1] = 1
    return mask


def interior(a, shape):
    """x = 1..nx-2: the reaction stage never touches the boundary planes, and
    the oracle reads their density as the prescribed boundary value"""
    a = np.asarray(a)
    return a.reshape(a.shape[:-1] + shape)[..., 1:-1, :, :]


def densities(t):
    return np.stack([t.density(s) for s in range(t.cfg.n_solutes)])


@pytest.mark.parametrize("gate", [True, False])
def test_kinetics_and_abiotic_stage_match_the_reference(pkg, gate):
    """Monod growth of two microbes (example 05) and Fe + HS -> FeS (example
    13) with and without the surface gate, one reaction stage."""
    need(13)
    nx, ny, nz = 14, 11, 9
    mask = geometry(nx, ny, nz, seed=2)
    rng = np.random.default_rng(7)
    sol = [{}, {}, {"immobile": True}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, microbes=2, dt=0.5)
    mu, Ks, Y, fP, kd = [2e-4, 1e-4], [5e-2, 5e-3], [0.4, 0.4], [2.0, 2.0], [1e-6, 1e-6]
    for m in range(2):
        pkg.add_rxn(cfg, microbe=m, k=mu[m], monod=[(0, Ks[m])], nu={0: -1.0 / Y[m], 1: fP[m]}, yield_=1.0)
        cfg.decay[m] = kd[m]
    pkg.add_rxn(cfg, k=20.0, mass=[0, 1], nu={0: -1.0, 1: -1.0, 2: 1.0})
    cfg.enable_kinetics = 1
    cfg.enable_abiotic = 1
    cfg.precip_enabled = 1 if gate else 0
    cfg.abiotic_surface_only = 1 if gate else 0
    N = mask.size
    C = np.stack([rng.uniform(0.0, 0.2, N), rng.uniform(0.0, 0.1, N), rng.uniform(0.0, 0.5, N)])
    B = np.where(rng.random((2, N)) < 0.3, rng.uniform(1.0, 50.0, (2, N)), 0.0)
    t = o.Transport(cfg, mask)
    for s in range(3):
        t.set_conc(s, C[s])
    for m in range(2):
        t.set_biomass(m, B[m])
    t.reaction_stage()
    flags = o.RXN_KINETICS | o.RXN_ABIOTIC | (o.RXN_SURFACE if gate else 0)
    rC, rB = o.ref_rxn_stage(13, cfg, mask, None, C, B, flags)
    oC = densities(t)
    assert np.abs(interior(oC - C, mask.shape)).max() > 1e-4       # the stage did something
    sh = mask.shape
    np.testing.assert_allclose(interior(oC, sh), interior(rC, sh), rtol=1e-10, atol=1e-14)
    np.testing.assert_allclose(interior(t.bio.reshape(2, N), sh), interior(rB, sh), rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize("with_abiotic", [True, False])
def test_dissolution_stage_matches_the_reference(pkg, with_abiotic):
    """Calcite dissolution of example 14 (rate k H mineral, H consumed, Ca
    released over the open faces, half-mineral cap), through the abiotic
    block or its own block (complab.cpp:1331-1366); the wall decrement
    dropped as the reference drops it."""
    need(14)
    nx, ny, nz = 14, 11, 9
    mask = geometry(nx, ny, nz, seed=4, grain_code=1)
    rng = np.random.default_rng(9)
    sol = [{}, {}, {"immobile": True}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, dt=1.0)
    cfg.dissol_enabled = 1
    cfg.reopen_fraction = 0.9
    cfg.dissol_surface_only = 1
    cfg.dissol_apply_at_walls = 0
    cfg.enable_abiotic = 1 if with_abiotic else 0
    pkg.add_phase(cfg, substrate=2, full_density=FULL, material=1, initial_fill=FULL,
                  k=1e-2, mass=[0], nu={0: -1.0, 1: 1.0})
    t = o.Transport(cfg, mask)
    N = mask.size
    C = np.stack([rng.uniform(1e-4, 1e-1, N), rng.uniform(0.0, 1e-3, N), t.imm[2 * N:3 * N].copy()])
    for s in range(2):
        t.set_conc(s, C[s])
    t.reaction_stage()
    flags = (o.RXN_ABIOTIC if with_abiotic else 0) | o.RXN_DISSOLUTION
    rC, _ = o.ref_rxn_stage(14, cfg, mask, t.phase, C, np.zeros((1, N)), flags)
    oC = densities(t)
    sh = mask.shape
    assert np.abs(interior(oC[1] - C[1], sh)).max() > 1e-4          # calcium released
    np.testing.assert_allclose(interior(oC, sh), interior(rC, sh), rtol=1e-10, atol=1e-14)


@pytest.mark.parametrize("solver", [0, 1])
def test_equilibrium_stage_matches_the_reference(pkg, solver):
    """run_equilibrium_biotic on example 04's carbonate tableau: the
    reference's PCF + Anderson solve and its 10% / 1e-9 step limiter against
    the oracle with the same limiter and Newton (rel 1e-6, both to a 1e-10
    residual) or the restated PCF + Anderson: the reference reads each
    concentration back from seven populations (~1e-16 absolute rounding), and
    a solve that stops at ||f||_2 < 1e-10 (f a log10 ratio) fixes the species
    to ln(10) * 1e-10 relative, so rel 5e-10 + abs 1e-14."""
    need(13)
    nx, ny, nz = 10, 8, 6
    mask = geometry(nx, ny, nz, seed=6)
    rng = np.random.default_rng(3)
    cfg = pkg.make_config(nx, ny, nz, solutes=[{}, {}, {}, {}])
    cfg.use_equilibrium = 1
    S = np.array([[1, 0], [0, 1], [1, -1], [1, 1]], float)
    pkg.set_eq_system(cfg.eq, S, [0.0, 0.0, -10.33, 6.35], [0, 1], max_iter=200, tol=1e-10, solver=solver)
    N = mask.size
    C = np.stack([rng.uniform(5e-4, 2e-3, N), 10 ** rng.uniform(-8, -6, N),
                  rng.uniform(1e-9, 1e-6, N), rng.uniform(1e-6, 1e-4, N)])
    t = o.Transport(cfg, mask)
    for s in range(4):
        t.set_conc(s, C[s])
    assert t.reaction_stage() == 0
    rC, _ = o.ref_rxn_stage(13, cfg, mask, None, C, np.zeros((1, N)), o.RXN_EQUILIBRIUM)
    oC = densities(t)
    sh = mask.shape
    moved = np.abs(interior(oC - C, sh)) > 1e-12
    assert moved.sum() > N // 2
    np.testing.assert_allclose(interior(oC, sh), interior(rC, sh), rtol=5e-10 if solver else 1e-6, atol=1e-14)


def test_node_conversions_match_the_reference(pkg):
    """precipNodeConversion3D (with phase stamping) and
    dissolNodeConversion3D on the same inventories: bit-exact masks and
    phases, the same counts."""
    need(13)
    need(14)
    nx, ny, nz = 12, 10, 8
    mask = geometry(nx, ny, nz, seed=8, grain_code=1)
    rng = np.random.default_rng(1)
    sol = [{}, {}, {"immobile": True}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol)
    cfg.precip_enabled = 1
    cfg.precip_substrate = 2
    cfg.max_precip_rho = 0.8
    cfg.precip_code = 0
    cfg.dissol_enabled = 1
    cfg.reopen_fraction = 0.9
    pkg.add_phase(cfg, substrate=2, full_density=FULL, material=1, initial_fill=FULL, k=0.0)
    pkg.add_phase(cfg, substrate=2, full_density=1.0, material=0, initial_fill=0.0, is_precipitate=True)
    cfg.precip_phase_id = 2
    t = o.Transport(cfg, mask)
    N = mask.size
    inv = t.imm[2 * N:3 * N]
    inv[:] = np.where(mask.reshape(-1) == 1, FULL * rng.uniform(0.85, 0.95, N), rng.uniform(0.0, 1.0, N))
    P = inv.copy()
    ch_ref, m_ref, ph_ref = o.ref_precip_convert(cfg, P, mask, t.phase)
    assert t.precip_convert() == ch_ref and ch_ref > 0
    np.testing.assert_array_equal(t.mask, m_ref)
    np.testing.assert_array_equal(t.phase, ph_ref)
    C = np.stack([np.zeros(N), np.zeros(N), inv.copy()])
    ch_ref, m_ref, ph_ref = o.ref_dissol_convert(cfg, C, t.mask, t.phase)
    assert t.dissol_convert() == ch_ref and ch_ref > 0
    np.testing.assert_array_equal(t.mask, m_ref)
    np.testing.assert_array_equal(t.phase, ph_ref)
