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


def test_surrogate_compiled_matches_table_and_oracle(gpu_lib, pkg, wl):
    """The surrogate workload's structure (six mobile solutes, two organisms
    with 3 -> 20 -> 20 -> 4 networks) runs its step in one launch with the
    networks' weights in the kernel's parameter space; the same fields as the
    run-time launches (rel. L2 <= 1e-12) and as the FP64 oracle."""
    mask = wl.sphere_pack(34, 20, 20, 0.40, 2.0, 4.0, seed=41)
    nx, ny, nz = mask.shape
    cfg = wl.surrogate_config(pkg, nx, ny, nz)
    nets = wl.surrogate_nets(pkg)
    bio = [wl.seed_biomass(mask, 42 + m, frac=0.3, lo=0.005, hi=0.05) for m in range(2)]

    def run(compiled, steps=30):
        lat = pkg.Lattice(cfg)
        lat.upload_mask(mask)
        lat.flow_init()
        lat.flow_steps(60)
        lat.couple_velocity()
        lat.set_option(pkg.OPT_COMPILED_CHEM, 1 if compiled else 0)
        for slot in range(2):
            lat.set_surrogate(slot, nets[slot])
        lat.ade_init()
        for m in range(2):
            lat.set_field(pkg.FIELD_BIOMASS, m, bio[m])
        for _ in range(steps):
            lat.step(1)
        out = {"conc": [lat.field(pkg.FIELD_CONC, s).reshape(-1) for s in range(cfg.n_solutes)],
               "bio": [lat.field(pkg.FIELD_BIOMASS, m).reshape(-1) for m in range(2)],
               "chem": lat.get_option(pkg.OPT_COMPILED_CHEM),
               "u": np.stack([lat.field(pkg.FIELD_VELOCITY, k).reshape(-1) for k in range(3)])}
        lat.close()
        return out

    fast, table = run(True), run(False)
    assert fast["chem"] == pkg.CHEM_SURROGATE2 and table["chem"] == 0
    for s in range(cfg.n_solutes):
        assert rel_l2(fast["conc"][s], table["conc"][s]) <= 1e-12, s
    for m in range(2):
        assert rel_l2(fast["bio"][m], table["bio"][m]) <= 1e-12, m
    tr = o.Transport(cfg, mask, u=fast["u"])
    tr.set_surrogates(nets)
    for m in range(2):
        tr.set_biomass(m, bio[m])
    tr.step(30)
    for s in range(cfg.n_solutes):
        assert rel_l2(fast["conc"][s], tr.density(s)) < 1e-4, s
    for m in range(2):
        assert rel_l2(fast["bio"][m], tr.biomass(m)) < 1e-5, m
    # a network of another shape: the step falls back to the run-time launches
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    odd = pkg.make_surrogate_net([3, 8, 4], [np.full((8, 3), 0.1), np.full((4, 8), 0.1)],
                                 [np.zeros(8), np.zeros(4)], np.zeros(3), np.ones(3), np.zeros(4), np.ones(4))
    lat.set_surrogate(0, odd)
    lat.set_surrogate(1, nets[1])
    lat.ade_init()
    assert lat.step(1) == pkg.OK
    lat.close()
