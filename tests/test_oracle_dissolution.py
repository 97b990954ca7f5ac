"""The oracle's dissolution processor on its own (CPU): element balance of the
release, the reference's dropped decrement on wall voxels, the half-mineral
cap, and reopening."""
import numpy as np
import pytest

from oracle import oracle as o


def cube_case(pkg, walls, k, fill=10.0, h=1e-2):
    """All-pore 12^3 domain with a 2^3 bounce-back cube in the middle carrying
    the phase; H+ uniform, no flow, Ca2+ zero."""
    nx = ny = nz = 12
    mask = np.full((nx, ny, nz), 2, np.uint8)
    mask[5:7, 5:7, 5:7] = 1
    sol = [{"tau": 0.8, "c0": h}, {"tau": 0.8, "c0": 0.0}, {"immobile": True, "c0": 0.0}]
    cfg = pkg.make_config(nx, ny, nz, solutes=sol, dt=1.0)
    cfg.dissol_enabled = 1
    cfg.reopen_fraction = 0.9
    cfg.dissol_surface_only = 1
    cfg.dissol_apply_at_walls = walls
    pkg.add_phase(cfg, substrate=2, full_density=fill, material=1, initial_fill=fill,
                  k=k, mass=[0], nu={0: -1.0, 1: 1.0})
    return cfg, mask


def total(ref, s):
    N = ref.N
    return ref.g[s * 7 * N:(s + 1) * 7 * N].sum()


def test_release_balances_the_mineral(pkg):
    cfg, mask = cube_case(pkg, walls=1, k=1e-2)
    ref = o.Transport(cfg, mask)
    m0 = ref.imm[2 * ref.N:3 * ref.N].sum()
    assert m0 == pytest.approx(8 * 10.0)
    ref.step(1)
    lost = m0 - ref.imm[2 * ref.N:3 * ref.N].sum()
    # each cube voxel has 3 open faces: water H = 1e-2, rate = k*H*mineral
    assert lost == pytest.approx(8 * 1e-2 * 1e-2 * 10.0, rel=1e-12)
    assert total(ref, 1) == pytest.approx(lost, rel=1e-12)


def test_wall_decrement_dropped_as_in_the_reference(pkg):
    cfg, mask = cube_case(pkg, walls=0, k=1e-2)
    ref = o.Transport(cfg, mask)
    ref.step(3)
    assert np.all(ref.imm[2 * ref.N:3 * ref.N][(mask == 1).reshape(-1)] == 10.0)
    assert total(ref, 1) > 0.0          # the products still reach the water


def test_half_mineral_cap(pkg):
    cfg, mask = cube_case(pkg, walls=1, k=1e6)
    ref = o.Transport(cfg, mask)
    ref.step(1)
    inv = ref.imm[2 * ref.N:3 * ref.N][(mask == 1).reshape(-1)]
    np.testing.assert_allclose(inv, 5.0, rtol=1e-15)
    # the products scale with the capped mineral loss
    assert total(ref, 1) == pytest.approx(8 * 5.0, rel=1e-12)


def test_reopening(pkg):
    cfg, mask = cube_case(pkg, walls=1, k=1e6)
    ref = o.Transport(cfg, mask)
    ref.step(1)                      # every cube voxel at half its fill
    assert ref.dissol_convert() == 8
    assert not ref.phase.any()
    assert np.all(ref.mask == 2)
    assert ref.dissol_convert() == 0
