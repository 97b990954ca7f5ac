"""The oracle's cellular-automaton biofilm on its own (CPU): mass balance and
the Bmax cap of pushExcessBiomass3D / halfPushExcessBiomass3D in both sweep
orders (the reference's in-place traversal and the plan-then-gather order the
CUDA library runs), the age wavefront of updateAgeDistance3D as a distance
transform, and the mask reclassification of updateLocalMaskNtotalLattices3D.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as o

BMAX = 1.0


def colony_case(pkg, half, shape=(18, 16, 14), seed=5, n_colonies=4, M=2):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    mask = np.full(shape, 2, np.uint8)
    mask[rng.random(shape) < 0.15] = 0
    mask[:, 0, :] = 1
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.8}], microbes=M, pore_codes=(2,), bio_codes=(3, 4))
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, half, BMAX, 0.1
    cfg.microbe_code[0], cfg.microbe_code[1] = 3, 4
    cfg.ca_seed = 2024
    bio = np.zeros((M,) + shape)
    for _ in range(n_colonies):
        x, y, z = rng.integers(2, nx - 2), rng.integers(2, ny - 1), rng.integers(0, nz)
        mask[x, y, z] = 3
        bio[0, x, y, z] = rng.uniform(3.0, 8.0)
        bio[1, x, y, z] = rng.uniform(0.0, 4.0)
    return cfg, mask, bio


def seeded(cfg, mask, bio):
    t = o.Transport(cfg, mask)
    for m in range(bio.shape[0]):
        t.set_biomass(m, bio[m])
    t.ca_init()
    return t


@pytest.mark.parametrize("half", [0, 1])
@pytest.mark.parametrize("serial", [False, True])
def test_mass_balance_and_cap(pkg, half, serial):
    cfg, mask, bio = colony_case(pkg, half)
    t = seeded(cfg, mask, bio)
    t.ca_update_mask()
    m0 = t.bio.sum()
    st, sweeps, changes, bmax = t.ca_redistribute(serial=serial)
    assert st == 0 and sweeps > 0 and changes > 0
    assert t.bio.sum() == pytest.approx(m0, rel=1e-13)
    tot = t.bio.reshape(2, -1).sum(0)
    assert tot.max() <= BMAX + 1e-12 and bmax == pytest.approx(tot.max(), rel=1e-15)
    np.testing.assert_allclose(t.ca_total, np.where(t.ca_total > 0, tot, 0.0), rtol=1e-12, atol=1e-12)
    # nothing moves into walls or outside x = 1..nx-2
    wall = np.isin(t.mask.reshape(cfg.nx, cfg.ny, cfg.nz), [0, 1]).reshape(-1)
    assert np.all(tot[wall] == 0.0)
    # reclassification: a pore voxel whose total reaches thrd * Bmax takes the
    # summed microbe codes of the species present; a biofilm voxel keeps its
    # code while it stays above the threshold
    bm = t.bio.reshape(2, -1)
    was_pore = (mask.reshape(-1) == 2)
    codes = 3 * (bm[0] > 1e-14) + 4 * (bm[1] > 1e-14)
    want = np.where(tot >= 0.1 * BMAX, np.where(was_pore, codes, mask.reshape(-1)), 2)
    open_ = ~wall
    np.testing.assert_array_equal(t.mask[open_], want[open_])


@pytest.mark.parametrize("half", [0, 1])
def test_orders_agree_statistically(pkg, half):
    """The two sweep orders spread the same colonies over about the same
    number of voxels in about the same number of sweeps."""
    out = {}
    for serial in (False, True):
        cfg, mask, bio = colony_case(pkg, half, shape=(24, 22, 20), n_colonies=10, seed=9)
        t = seeded(cfg, mask, bio)
        t.ca_update_mask()
        st, sweeps, _, _ = t.ca_redistribute(serial=serial)
        assert st == 0
        out[serial] = (sweeps, int(np.isin(t.mask, [3, 4, 7]).sum()))
    (s0, v0), (s1, v1) = out[False], out[True]
    assert abs(v0 - v1) <= max(3, 0.2 * v1), out
    assert 0.5 * s1 - 2 <= s0 <= 2 * s1 + 2, out


def test_age_wavefront_is_a_distance_transform(pkg):
    """A 7^3 block of biofilm at Bmax with a slight excess in its centre: the
    ages relax to 1 + the face distance to the block's surface (the wavefront
    of updateAgeDistance3D), and the excess leaves the block."""
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
    t = seeded(cfg, mask, bio)
    t.ca_update_mask()
    st, sweeps, _, _ = t.ca_redistribute()
    assert st == 0 and sweeps >= 4                 # the excess walks out through 3 full layers
    age = t.ca_age.reshape(n, n, n)
    idx = np.arange(lo, hi)
    d = np.minimum(idx - lo, hi - 1 - idx)
    layer = np.minimum(np.minimum(d[:, None, None], d[None, :, None]), d[None, None, :])
    np.testing.assert_array_equal(age[lo:hi, lo:hi, lo:hi], 1 + layer)
    tot = t.bio.reshape(n, n, n)
    assert np.all(tot[lo:hi, lo:hi, lo:hi] <= BMAX)
    assert tot.sum() - BMAX * 7 ** 3 == pytest.approx(1e-6, rel=1e-6)
    outside = tot.copy()
    outside[lo:hi, lo:hi, lo:hi] = 0.0
    assert outside.sum() == pytest.approx(1e-6, rel=1e-6)


def test_boxed_in_voxel_keeps_its_excess(pkg):
    """A voxel whose face neighbours are all walls cannot push (the
    reference's [CA-ROBUST] branch) and its age has no neighbour to stop it,
    so the first age relaxation runs into its 1000-pass limit: the block ends
    after one sweep with the not-converged status (the reference ends the run
    there) and the excess stays where it is."""
    n = 9
    cfg = pkg.make_config(n, n, n, solutes=[{"tau": 0.8}], microbes=1, pore_codes=(2,), bio_codes=(3,))
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, 0, BMAX, 0.1
    cfg.microbe_code[0] = 3
    mask = np.full((n, n, n), 2, np.uint8)
    mask[3:6, 3:6, 3:6] = 0
    mask[4, 4, 4] = 3
    bio = np.zeros((1, n, n, n))
    bio[0, 4, 4, 4] = 2.5
    t = seeded(cfg, mask, bio)
    st, sweeps, _, bmax = t.ca_redistribute()
    assert st == 1 and sweeps == 1 and bmax == 2.5
    assert t.bio.reshape(n, n, n)[4, 4, 4] == 2.5
    assert t.ca_age.reshape(n, n, n)[4, 4, 4] > 1000


def _pin_case(pkg, half, M, n_pore, seed):
    """Dyadic biomass (exact in the reference's (d-1)/4, (d-1)/8 population
    encoding) on a walled channel with cube grains and colonies away from the
    x boundary planes.  With the half push both microbes get the same density:
    a voxel at Bmax pushes half its biomass or nothing depending on the last
    bit of its total, so shares that stop being dyadic would make the two
    codes' rounding, not their logic, decide."""
    nx, ny, nz = 16, 13, 11
    rng = np.random.default_rng(seed)
    pores = (2, 5) if n_pore == 2 else (2,)
    mask = np.full((nx, ny, nz), 2, np.uint8)
    if n_pore == 2:
        mask[:, :, nz // 2:] = 5
    for _ in range(6):
        x, y, z = rng.integers(1, nx - 4), rng.integers(1, ny - 4), rng.integers(1, nz - 4)
        mask[x:x + 2, y:y + 2, z:z + 2] = 0
    mask[:, 0, :] = mask[:, ny - 1, :] = 1
    mask[:, :, 0] = mask[:, :, nz - 1] = 1
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.8}], microbes=M, pore_codes=pores, bio_codes=(3, 4))
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, half, 1.0, 0.1
    cfg.microbe_code[0] = 3
    if M > 1:
        cfg.microbe_code[1] = 4
    cfg.ca_seed = 4321 + seed
    bio = np.zeros((M, nx, ny, nz))
    placed = 0
    while placed < 10:
        x, y, z = rng.integers(3, nx - 3), rng.integers(1, ny - 1), rng.integers(1, nz - 1)
        if mask[x, y, z] in (2, 5):
            mask[x, y, z] = 3
            v = rng.integers(1, 48) / 8.0
            for m in range(M):
                bio[m, x, y, z] = v if half else rng.integers(1, 48) / 8.0
            placed += 1
    return cfg, mask, bio


@pytest.mark.parametrize("half,M,n_pore", [(0, 1, 1), (1, 1, 1), (0, 2, 1), (1, 2, 1), (0, 1, 2)])
def test_serial_order_matches_the_reference_processors(pkg, half, M, n_pore):
    """The oracle's serial order against the reference's own
    updateLocalMaskNtotalLattices3D / push / updateAgeDistance3D processors,
    compiled from its sources and run on one block with the same draws: the
    same sweeps, masks and ages, and biomass equal to 1e-13 (the reference
    keeps biomass as seven populations, which round differently from one
    FP64 value once shares stop being dyadic)."""
    if o.ref_lib() is None:
        pytest.skip("reference tree absent: oracle/_ref not built")
    cfg, mask, bio = _pin_case(pkg, half, M, n_pore, seed=3 * half + M + 5 * n_pore)
    t = seeded(cfg, mask, bio)
    r = o.RefCa(cfg, mask, bio, t.ca_distpos, total=t.ca_total, age=t.ca_age, mask_sum=int(t.ca.mask_sum))
    assert t.ca_update_mask(serial=True) == r.update_mask()
    rng = np.random.default_rng(11)
    for block in range(3):
        st, sweeps, _, gmax = t.ca_redistribute(serial=True)
        rst, rsweeps, rgmax = r.block()
        assert (st, sweeps) == (rst, rsweeps), block
        assert sweeps > 0
        assert gmax == pytest.approx(rgmax, rel=1e-13)
        np.testing.assert_array_equal(t.mask, r.mask)
        np.testing.assert_array_equal(t.ca_age, r.age)
        np.testing.assert_allclose(t.bio[:M * t.N], r.bio, rtol=1e-13, atol=1e-13)
        np.testing.assert_allclose(t.ca_total, r.total, rtol=1e-13, atol=1e-13)
        assert t.ca.draws == r.draws.value
        # dyadic growth between blocks, the same on both sides
        g = rng.integers(9, 16, size=t.N) / 8.0
        for m in range(M):
            b = t.biomass(m) * g
            t.set_biomass(m, b)
            r.bio[m * t.N:(m + 1) * t.N] = b


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_fd_diffusion_matches_the_reference_processor(pkg, seed):
    """The finite-difference biomass step (solver_type FD) against the
    reference's own fdDiffusion3D, compiled from its sources and run on one
    block: random biomass (some of it below thrd) of two microbes, one of
    them selected, on a channel walled in y and z with cube grains, so the
    no-flux sides, the x-planes left out and the thresholds all occur.  Equal
    to 1e-13 (the reference stores each value as seven populations)."""
    if o.ref_lib() is None:
        pytest.skip("reference tree absent: oracle/_ref not built")
    nx, ny, nz = 14, 11, 9
    rng = np.random.default_rng(seed)
    mask = np.full((nx, ny, nz), 2, np.uint8)
    for _ in range(5):
        x, y, z = rng.integers(1, nx - 3), rng.integers(1, ny - 3), rng.integers(1, nz - 3)
        mask[x:x + 2, y:y + 2, z:z + 2] = 0
    mask[:, 0, :] = mask[:, ny - 1, :] = 1
    mask[:, :, 0] = mask[:, :, nz - 1] = 1
    mask[(mask == 2) & (rng.random(mask.shape) < 0.3)] = 3
    M = 2
    bio = rng.random((M, nx, ny, nz)) * (rng.random((M, nx, ny, nz)) < 0.7)
    bio[bio < 0.05] *= 1e-15                      # some values below thrd
    bio[:, mask <= 1] = 0.0
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.8}], microbes=M, bio_codes=(3,))
    t = o.Transport(cfg, mask.reshape(-1))
    for m in range(M):
        t.set_biomass(m, bio[m].reshape(-1))
    nu = 0.13
    t.fd_diffuse(nu, 0b01)
    ref = np.ascontiguousarray(bio.reshape(-1), np.float64).copy()
    o.ref_lib().ref_fd_diffuse(ctypes.c_int(nx), ctypes.c_int(ny), ctypes.c_int(nz), ctypes.c_int(1),
                               ctypes.c_double(nu), np.ascontiguousarray(mask.reshape(-1)).ctypes.data_as(ctypes.c_void_p),
                               ref.ctypes.data_as(ctypes.c_void_p))
    N = nx * ny * nz
    np.testing.assert_allclose(t.biomass(0), ref[:N], rtol=1e-13, atol=1e-13)
    assert np.abs(t.biomass(0) - bio[0].reshape(-1)).max() > 1e-3       # it did diffuse
    np.testing.assert_array_equal(t.biomass(1), bio[1].reshape(-1))      # not selected
