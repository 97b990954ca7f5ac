"""The learned warm start inside the transport step (CL_OPT_EQ_LEARN): the
network is trained on the device during the run on the pairs the step's own
Newton solves produce, and gives the start of every voxel that has no
previous solution of its own.

Two contexts run the benchmark's coupled chemistry (256x128x128 sphere pack,
mineral coatings, dissolution) from the same state, one learning (training
every 10 steps on 1/16 of the converged voxels' pairs) and one not.  After 40
steps both forget their previous solutions and take one more step: the
learning one starts each voxel from the network where its guess has the
smaller mass-balance residual, the other from the reference's cold start.
Newton's 1e-10 relative residual decides convergence in both, so the fields
agree to rel. L2 <= 1e-6, and the learned start needs fewer Newton iterations
per reactive voxel."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def test_learned_start_in_the_step(gpu_lib, pkg, wl):
    shape = (256, 128, 128)
    mask = wl.sphere_pack(*shape, 0.35, 5.0, 10.0, seed=15)
    cfg = wl.coupled_config(pkg, *shape, dissolution=True)
    bio = wl.seed_biomass(mask, 16)
    mineral = wl.seed_mineral(mask, 17, cfg.max_precip_rho)
    react = (mask == 2)
    react[0] = react[-1] = False
    react = react.reshape(-1)
    out = {}
    for learn in (True, False):
        lat = pkg.Lattice(cfg)
        lat.upload_mask(mask)
        lat.flow_init()
        lat.flow_steps(100)
        lat.couple_velocity()
        lat.ade_init()
        lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
        lat.set_field(pkg.FIELD_CONC, 8, mineral)
        if learn:
            lat.set_option(pkg.OPT_EQ_LEARN, 10)
        for _ in range(40):
            assert lat.step(1) == pkg.OK
        if learn:
            assert lat.get_option(pkg.OPT_EQ_LEARN_TRAININGS) >= 3
        lat.set_option(pkg.OPT_EQ_FORGET, 1)
        assert lat.step(1) == pkg.OK
        it = lat.field(pkg.FIELD_EQ_ITERS).reshape(-1)[react]
        out[learn] = ([lat.field(pkg.FIELD_CONC, s).reshape(-1) for s in range(cfg.n_solutes)], float(it.mean()))
        lat.close()
    for s in range(cfg.n_solutes):
        assert rel_l2(out[True][0][s], out[False][0][s]) <= 1e-6, s
    path = os.environ.get("COMPLAB_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"case": "learned start in the step", "iters_learned": out[True][1],
                                "iters_cold": out[False][1]}) + "\n")
    assert out[True][1] < out[False][1], (out[True][1], out[False][1])
