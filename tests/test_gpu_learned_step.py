"""The learned warm start inside the transport step (CL_OPT_EQ_LEARN): the
network is trained on the device during the run on the pairs the step's own
Newton solves produce, and gives the start of every voxel that has no
previous solution of its own.

Two contexts run the coupled chemistry from the same state, one learning
(training every 5 steps) and one not.  After 20 steps both forget their
previous solutions, their carbonate water is replaced by the same unspeciated
water (every component at its total in its own species, the complexes empty:
water as it enters, or as a reopened voxel holds it) and they take one more
step: the learning one starts from the network where its guess has the
smaller mass-balance residual, the other from the reference's cold start.
Newton's 1e-10 relative residual decides convergence in both, so the fields
agree to rel. L2 <= 1e-6, and the learned start needs fewer iterations per
voxel."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def test_learned_start_in_the_step(gpu_lib, pkg, wl):
    mask = wl.sphere_pack(66, 32, 32, 0.45, 2.0, 4.0, seed=71)
    nx, ny, nz = mask.shape
    cfg = wl.coupled_config(pkg, nx, ny, nz)
    bio = wl.seed_biomass(mask, 72, frac=0.2)
    out = {}
    for learn in (True, False):
        lat = pkg.Lattice(cfg)
        lat.upload_mask(mask)
        lat.flow_init()
        lat.flow_steps(100)
        lat.couple_velocity()
        lat.ade_init()
        lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
        if learn:
            lat.set_option(pkg.OPT_EQ_LEARN, 5)
        for _ in range(20):
            assert lat.step(1) == pkg.OK
        if learn:
            assert lat.get_option(pkg.OPT_EQ_LEARN_TRAININGS) >= 2
        lat.set_option(pkg.OPT_EQ_FORGET, 1)
        # unspeciated: HCO3- (3) = CO3-- + H+, CaCO3 (7) = CO3-- + Ca++ back
        # into their components CO3-- (6), Ca++ (4), H+ (5)
        c = {sp: lat.field(pkg.FIELD_CONC, sp) for sp in (3, 4, 5, 6, 7)}
        lat.set_field(pkg.FIELD_CONC, 6, c[6] + c[3] + c[7])
        lat.set_field(pkg.FIELD_CONC, 4, c[4] + c[7])
        lat.set_field(pkg.FIELD_CONC, 5, c[5] + c[3])
        lat.set_field(pkg.FIELD_CONC, 3, np.zeros_like(c[3]))
        lat.set_field(pkg.FIELD_CONC, 7, np.zeros_like(c[7]))
        # from water this far from equilibrium a few voxels may miss the
        # tolerance (and keep their state, as the reference's Newton does)
        assert lat.step(1) in (pkg.OK, pkg.WARN_NOT_CONVERGED)
        react = (mask == 2).reshape(-1)
        it = lat.field(pkg.FIELD_EQ_ITERS).reshape(-1)
        out[learn] = ([lat.field(pkg.FIELD_CONC, s).reshape(-1) for s in range(cfg.n_solutes)], it[react].mean(), it)
        lat.close()
    # a voxel that missed the tolerance in either run kept its water there
    # (and streamed it to its face neighbours): those are left out
    miss = ((out[True][2] >= cfg.eq.max_iter) | (out[False][2] >= cfg.eq.max_iter)).reshape(mask.shape)
    near = miss.copy()
    for ax in range(3):
        for sh in (1, -1):
            near |= np.roll(miss, sh, axis=ax)
    keep = ~near.reshape(-1)
    assert keep.mean() > 0.99
    for s in range(cfg.n_solutes):
        assert rel_l2(out[True][0][s][keep], out[False][0][s][keep]) <= 1e-6, s
    path = os.environ.get("COMPLAB_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"case": "learned start in the step", "iters_learned": float(out[True][1]),
                                "iters_cold": float(out[False][1])}) + "\n")
    assert out[True][1] < out[False][1], (out[True][1], out[False][1])
