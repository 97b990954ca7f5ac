"""The one-launch transport step of a compiled chemistry against the
run-time-table launches and the FP64 oracle.

A configuration whose structure matches a chemistry compiled into the library
(the coupled carbonate chemistry, the biotic dual-Monod chemistry) runs its
transport step in one launch with every voxel's state in registers.  Its
arithmetic is that of the run-time-table launches operation for operation:
the fields of the two agree to rel. L2 <= 1e-12 (FP64 chain; the FP32
populations see the same increments), and both agree with the FP64 oracle to
the transport tolerance, rel. L2 <= 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _run(pkg, cfg, mask, bio, steps, compiled, flow_steps=60, variant=0):
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(flow_steps)
    lat.couple_velocity()
    lat.set_option(pkg.OPT_COMPILED_CHEM, 1 if compiled else 0)
    lat.set_option(pkg.OPT_FAST_VARIANT, variant)
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
    for _ in range(steps):
        lat.step(1)
    out = {"conc": [lat.field(pkg.FIELD_CONC, s).reshape(-1) for s in range(cfg.n_solutes)],
           "bio": lat.field(pkg.FIELD_BIOMASS, 0).reshape(-1),
           "chem": lat.get_option(pkg.OPT_COMPILED_CHEM),
           "u": np.stack([lat.field(pkg.FIELD_VELOCITY, k).reshape(-1) for k in range(3)])}
    if cfg.use_equilibrium:
        out["iters"] = lat.field(pkg.FIELD_EQ_ITERS).reshape(-1)
    lat.close()
    return out


# launch shapes of the one-launch step: 0 128 threads x 4 blocks per SM,
# 2 64 x 6 (a different register cap, so different code)
@pytest.mark.parametrize("variant", [0, 2])
@pytest.mark.parametrize("steps", [1, 2, 25])
def test_coupled_compiled_matches_table_and_oracle(gpu_lib, pkg, wl, steps, variant):
    mask = wl.sphere_pack(34, 16, 16, 0.45, 2.0, 4.0, seed=3)
    nx, ny, nz = mask.shape
    cfg = wl.coupled_config(pkg, nx, ny, nz, dissolution=True)
    bio = wl.seed_biomass(mask, 4, frac=0.3)
    fast = _run(pkg, cfg, mask, bio, steps, True, variant=variant)
    table = _run(pkg, cfg, mask, bio, steps, False)
    assert fast["chem"] == pkg.CHEM_COUPLED and table["chem"] == 0
    for s in range(cfg.n_solutes):
        assert rel_l2(fast["conc"][s], table["conc"][s]) <= 1e-12, s
    assert rel_l2(fast["bio"], table["bio"]) <= 1e-12
    assert np.array_equal(fast["iters"], table["iters"])
    tr = o.Transport(cfg, mask, u=fast["u"])
    tr.set_biomass(0, bio)
    tr.step(steps)
    for s in range(cfg.n_solutes):
        assert rel_l2(fast["conc"][s], tr.density(s)) < 1e-4, s
    assert rel_l2(fast["bio"], tr.biomass(0)) < 1e-5


@pytest.mark.parametrize("variant", [0, 2])
def test_biotic_compiled_matches_table_and_oracle(gpu_lib, pkg, wl, variant):
    mask = wl.sphere_pack(30, 16, 16, 0.4, 2.0, 4.0, seed=8)
    nx, ny, nz = mask.shape
    cfg = wl.biotic_config(pkg, nx, ny, nz)
    cfg.ca_enabled = 0
    cfg.dt = 50.0
    bio = wl.seed_biomass(mask, 9, frac=0.3)
    fast = _run(pkg, cfg, mask, bio, 30, True, variant=variant)
    table = _run(pkg, cfg, mask, bio, 30, False)
    assert fast["chem"] == pkg.CHEM_BIOTIC4 and table["chem"] == 0
    for s in range(cfg.n_solutes):
        assert rel_l2(fast["conc"][s], table["conc"][s]) <= 1e-12, s
    assert rel_l2(fast["bio"], table["bio"]) <= 1e-12
    tr = o.Transport(cfg, mask, u=fast["u"])
    tr.set_biomass(0, bio)
    tr.step(30)
    for s in range(cfg.n_solutes):
        assert rel_l2(fast["conc"][s], tr.density(s)) < 1e-4, s
    assert rel_l2(fast["bio"], tr.biomass(0)) < 1e-5
