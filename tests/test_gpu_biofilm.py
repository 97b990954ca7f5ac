"""Cellular-automaton biofilm on the GPU (cl_ca_update_mask /
cl_ca_redistribute) against the FP64 oracle in the same plan-then-gather
sweep order.

The CA is FP64 bookkeeping with a counter-based generator, so the bar is
bit-exact: biomass, total, mask and age fields equal, and the same sweep
and mask-change counts.  At a larger size the invariants are checked
instead: the biomass sum is conserved to 1e-12 relative and no voxel ends
above Bmax.
"""
import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu

BMAX = 1.0


def colony_case(pkg, half, shape, seed, n_colonies, M=2):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    mask = np.full(shape, 2, np.uint8)
    # solid grains as 3^3 cubes in a channel with bounce-back walls on the
    # four y / z faces: the pore space stays connected and no biomass reaches
    # the last y or z index.  A full colony sealed in, or a biofilm voxel on a
    # last index whose neighbours are all off the reference's distance field,
    # has an age that never settles, and the block then ends with the
    # not-converged status, as the reference's run ends.
    for _ in range(int(0.05 * nx * ny * nz / 27) + 1):
        x, y, z = rng.integers(0, nx - 2), rng.integers(0, ny - 2), rng.integers(0, nz - 2)
        mask[x:x + 3, y:y + 3, z:z + 3] = 0
    mask[:, 0, :] = mask[:, ny - 1, :] = 1
    mask[:, :, 0] = mask[:, :, nz - 1] = 1
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.8}], microbes=M, pore_codes=(2,), bio_codes=(3, 4))
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, half, BMAX, 0.1
    cfg.microbe_code[0], cfg.microbe_code[1] = 3, 4
    cfg.ca_seed = 77 + half
    bio = np.zeros((M,) + shape)
    for _ in range(n_colonies):
        x, y, z = rng.integers(1, nx - 1), rng.integers(0, ny), rng.integers(0, nz)
        if mask[x, y, z] in (0, 1):
            continue
        mask[x, y, z] = 3
        bio[0, x, y, z] = rng.uniform(2.0, 9.0)
        bio[1, x, y, z] = rng.uniform(0.0, 3.0)
    return cfg, mask, bio


def both(pkg, cfg, mask, bio):
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    ref = o.Transport(cfg, mask)
    for m in range(bio.shape[0]):
        lat.set_field(pkg.FIELD_BIOMASS, m, bio[m])
        ref.set_biomass(m, bio[m])
    ref.ca_init()
    return lat, ref


def assert_same(pkg, lat, ref, M):
    for m in range(M):
        np.testing.assert_array_equal(lat.field(pkg.FIELD_BIOMASS, m).reshape(-1), ref.biomass(m), err_msg="bio%d" % m)
    np.testing.assert_array_equal(lat.mask().reshape(-1), ref.mask)
    np.testing.assert_array_equal(lat.field(pkg.FIELD_CA_TOTAL).reshape(-1), ref.ca_total)
    np.testing.assert_array_equal(lat.field(pkg.FIELD_CA_AGE).reshape(-1), ref.ca_age.astype(float))


@pytest.mark.parametrize("half", [0, 1])
def test_ca_matches_oracle_bit_exact(gpu_lib, pkg, half):
    shape = (26, 21, 17)
    cfg, mask, bio = colony_case(pkg, half, shape, seed=11 + half, n_colonies=14)
    lat, ref = both(pkg, cfg, mask, bio)
    np.testing.assert_array_equal(lat.field(pkg.FIELD_CA_AGE).reshape(-1), ref.ca_age.astype(float))
    assert lat.ca_update_mask() == ref.ca_update_mask()
    assert_same(pkg, lat, ref, 2)
    rng = np.random.default_rng(5)
    for block in range(4):
        got = lat.ca_redistribute()
        want = ref.ca_redistribute()
        assert got == want, (block, got, want)
        assert got[1] > 0
        assert_same(pkg, lat, ref, 2)
        # growth between blocks, the same on both sides
        g = rng.uniform(1.2, 1.8, size=(2,) + shape)
        for m in range(2):
            b = ref.biomass(m).reshape(shape) * g[m]
            lat.set_field(pkg.FIELD_BIOMASS, m, b)
            ref.set_biomass(m, b)


def test_ca_age_distance_transform(gpu_lib, pkg):
    """A 7^3 biofilm block at Bmax with a slight excess at its centre: the
    ages relax to 1 + the face distance to the block's surface."""
    n = 15
    cfg = pkg.make_config(n, n, n, solutes=[{"tau": 0.8}], microbes=1, pore_codes=(2,), bio_codes=(3,))
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, 0, BMAX, 0.1
    cfg.microbe_code[0] = 3
    cfg.ca_seed = 1
    mask = np.full((n, n, n), 2, np.uint8)
    lo, hi = 4, 11
    mask[lo:hi, lo:hi, lo:hi] = 3
    bio = np.zeros((1, n, n, n))
    bio[0, lo:hi, lo:hi, lo:hi] = BMAX
    bio[0, 7, 7, 7] = BMAX + 1e-6
    lat, ref = both(pkg, cfg, mask, bio)
    lat.ca_update_mask()
    ref.ca_update_mask()
    assert lat.ca_redistribute() == ref.ca_redistribute()
    age = lat.field(pkg.FIELD_CA_AGE)
    idx = np.arange(lo, hi)
    d = np.minimum(idx - lo, hi - 1 - idx)
    layer = np.minimum(np.minimum(d[:, None, None], d[None, :, None]), d[None, None, :])
    np.testing.assert_array_equal(age[lo:hi, lo:hi, lo:hi], 1 + layer)
    assert_same(pkg, lat, ref, 1)


@pytest.mark.parametrize("half", [0, 1])
def test_ca_invariants_large(gpu_lib, pkg, half):
    shape = (192, 128, 128)
    cfg, mask, bio = colony_case(pkg, half, shape, seed=3, n_colonies=4000)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    for m in range(2):
        lat.set_field(pkg.FIELD_BIOMASS, m, bio[m])
    m0 = bio.sum()
    lat.ca_update_mask()
    st, sweeps, changes, bmax = lat.ca_redistribute()
    assert st == 0 and sweeps > 0 and changes > 0
    tot = lat.field(pkg.FIELD_BIOMASS, 0) + lat.field(pkg.FIELD_BIOMASS, 1)
    assert tot.sum() == pytest.approx(m0, rel=1e-12)
    assert tot.max() <= BMAX + 1e-12 and bmax <= BMAX + 1e-12
    wall = np.isin(lat.mask(), [0, 1])
    assert np.all(tot[wall] == 0.0)


@pytest.mark.parametrize("seed", [1, 2])
def test_fd_diffusion_matches_oracle_bit_for_bit(gpu_lib, pkg, seed):
    """The finite-difference biomass step on the GPU (fd_diffuse_kernel)
    against the oracle, which the reference's own fdDiffusion3D pins
    (test_oracle_biofilm.py): the same FP64 sums in the same order, so the
    biomass fields are equal bit for bit, over three steps with the
    mask update between them."""
    nx, ny, nz = 30, 17, 13
    rng = np.random.default_rng(seed)
    mask = np.full((nx, ny, nz), 2, np.uint8)
    for _ in range(12):
        x, y, z = rng.integers(1, nx - 3), rng.integers(1, ny - 3), rng.integers(1, nz - 3)
        mask[x:x + 2, y:y + 2, z:z + 2] = 0
    mask[:, 0, :] = mask[:, ny - 1, :] = 1
    mask[:, :, 0] = mask[:, :, nz - 1] = 1
    mask[(mask == 2) & (rng.random(mask.shape) < 0.3)] = 3
    M = 2
    bio = rng.random((M, nx, ny, nz)) * 40.0 * (rng.random((M, nx, ny, nz)) < 0.6)
    bio[:, mask <= 1] = 0.0
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.8}], microbes=M, bio_codes=(3,))
    cfg.ca_enabled, cfg.ca_bmax, cfg.ca_thrd_frac = 1, 50.0, 0.01
    cfg.microbe_code[0] = cfg.microbe_code[1] = 3
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.ade_init()
    t = o.Transport(cfg, mask.reshape(-1))
    t.ca_init()
    for m in range(M):
        lat.set_field(pkg.FIELD_BIOMASS, m, bio[m])
        t.set_biomass(m, bio[m].reshape(-1))
    for k in range(3):
        ch = lat.ca_update_mask()
        assert ch == t.ca_update_mask()
        lat.fd_diffuse(0.05, 0b11)
        t.fd_diffuse(0.05, 0b11)
        for m in range(M):
            np.testing.assert_array_equal(lat.field(pkg.FIELD_BIOMASS, m).reshape(-1), t.biomass(m), err_msg=str((k, m)))
        np.testing.assert_array_equal(lat.mask().reshape(-1), t.mask)
    lat.close()
