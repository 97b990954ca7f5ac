"""Mineral dissolution (surfaceDissolutionKinetics3D) and pore reopening
(dissolNodeConversion3D) on the GPU against the FP64 oracle.

Tolerances as for the other reaction tests: solute fields relative L2 <= 1e-4;
the mineral's loss (inventory minus its seed) relative L2 <= 1e-4; phase and
mask fields bit-exact.
"""
import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


FULL = 27.1      # mol/L in a full calcite voxel (1000 / 36.9 cm3/mol)


def calcite_config(pkg, shape, walls, k=2e-3, dt=1.0):
    """Example 14's chemistry: H+ (0) enters from the left, Ca2+ (1) is
    released, calcite (2) is the immobile inventory of the grain phase, which
    occupies the grains' surface voxels (material 1)."""
    nx, ny, nz = shape
    sol = [{"tau": 0.8, "c0": 1e-4, "left": "D", "left_value": 1e-2, "right": "N"},
           {"tau": 0.8, "c0": 0.0, "left": "N", "right": "N"},
           {"immobile": True, "c0": 0.0}]
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.0005, rho_out=1.0, solutes=sol, dt=dt)
    cfg.dissol_enabled = 1
    cfg.reopen_fraction = 0.9
    cfg.dissol_surface_only = 1
    cfg.dissol_apply_at_walls = walls
    pkg.add_phase(cfg, substrate=2, full_density=FULL, material=1, initial_fill=FULL,
                  k=k, mass=[0], nu={0: -1.0, 1: 1.0})
    return cfg


def flow_field(pkg, cfg, mask, steps=200):
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(steps)
    lat.couple_velocity()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, k).reshape(-1) for k in range(3)])
    return lat, u


@pytest.mark.parametrize("walls", [0, 1])
def test_calcite_dissolution_and_reopening(gpu_lib, pkg, wl, walls):
    mask = wl.sphere_pack(20, 14, 14, 0.55, 2.0, 3.5, seed=31)
    cfg = calcite_config(pkg, mask.shape, walls)
    lat, u = flow_field(pkg, cfg, mask)
    lat.ade_init()
    ref = o.Transport(cfg, mask, u=u)
    # the phase lattice and the grain inventories are seeded from the geometry
    np.testing.assert_array_equal(lat.field(pkg.FIELD_PHASE).reshape(-1), ref.phase.astype(float))
    assert (ref.phase == 1).sum() == (mask == 1).sum()
    for n in (1, 4, 35):
        lat.step(n)
        ref.step(n)
    for s in range(2):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    ca = ref.density(1)
    assert ca.max() > 1e-3                                       # dissolution released calcium
    mg, mo = lat.field(pkg.FIELD_CONC, 2).reshape(-1), ref.density(2)
    grain = (mask == 1).reshape(-1)
    if walls:
        lost_o = FULL - mo[grain]
        assert lost_o.max() > 0
        assert rel_l2(FULL - mg[grain], lost_o) < 1e-4
    else:
        # the reference drops a decrement written on a bounce-back voxel
        assert np.all(mg[grain] == FULL) and np.all(mo[grain] == FULL)
    # reopening, bit-exact given the same inventories
    rng = np.random.default_rng(3)
    inv = mo.copy()
    inv[grain] = FULL * rng.uniform(0.85, 0.95, int(grain.sum()))
    lat.set_field(pkg.FIELD_CONC, 2, inv)
    ref.imm[2 * ref.N:3 * ref.N] = inv
    ch_g, ch_o = lat.dissol_convert(), ref.dissol_convert()
    assert ch_g == ch_o and 0 < ch_o < int(grain.sum())
    np.testing.assert_array_equal(lat.mask().reshape(-1), ref.mask)
    np.testing.assert_array_equal(lat.field(pkg.FIELD_PHASE).reshape(-1), ref.phase.astype(float))
    # reopened voxels react again (their solute dynamics stay as they were)
    lat.step(10)
    ref.step(10)
    for s in range(3):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    lat.close()


def test_precipitate_then_dissolve(gpu_lib, pkg, wl):
    """Example 15: Fe + HS -> FeS(s) on wall-adjacent voxels; sealed voxels are
    stamped with the precipitate phase, which acid then dissolves back."""
    mask = wl.sphere_pack(20, 14, 14, 0.55, 2.0, 3.0, seed=13)
    nx, ny, nz = mask.shape
    sol = [{"tau": 0.8, "c0": 0.5, "left": "D", "left_value": 5.0, "right": "N"},
           {"tau": 0.8, "c0": 0.5, "left": "N", "right": "D", "right_value": 5.0},
           {"tau": 0.8, "c0": 1e-3, "left": "D", "left_value": 1e-2, "right": "N"},
           {"immobile": True, "c0": 0.0}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, dt=0.01)
    cfg.enable_abiotic = 1
    cfg.precip_enabled = 1
    cfg.abiotic_surface_only = 1
    cfg.precip_substrate = 3
    cfg.max_precip_rho = 0.8
    cfg.precip_code = 0
    pkg.add_rxn(cfg, k=20.0, mass=[0, 1], nu={0: -1.0, 1: -1.0, 3: 1.0})
    cfg.dissol_enabled = 1
    cfg.reopen_fraction = 0.9
    cfg.dissol_surface_only = 1
    cfg.dissol_apply_at_walls = 1
    pkg.add_phase(cfg, substrate=3, full_density=0.8, is_precipitate=True,
                  k=50.0, mass=[2], nu={0: 1.0, 1: 1.0, 2: -1.0})
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    ref = o.Transport(cfg, mask)
    assert not ref.phase.any() and not lat.field(pkg.FIELD_PHASE).any()
    lat.step(60)
    ref.step(60)
    for s in range(4):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    inv = ref.density(3)
    lat.set_field(pkg.FIELD_CONC, 3, inv)
    ch_g, ch_o = lat.precip_convert(), ref.precip_convert()
    assert ch_g == ch_o and ch_o > 0
    np.testing.assert_array_equal(lat.mask().reshape(-1), ref.mask)
    np.testing.assert_array_equal(lat.field(pkg.FIELD_PHASE).reshape(-1), ref.phase.astype(float))
    # the sealed voxels now dissolve at their wetted faces
    sealed = ref.phase == 1
    before = inv[sealed].copy()
    lat.step(40)
    ref.step(40)
    for s in range(4):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), ref.density(s)) < 1e-4, s
    assert (ref.density(3)[sealed] < before).any()
    lat.close()
