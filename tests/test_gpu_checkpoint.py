"""Checkpoint and restart through the C ABI: the state a transport step reads
(dynamics classes, flow and solute populations in natural order, immobile
inventories, biomass, phase ids, the Newton warm starts) taken from one context after 5 steps of
the coupled chemistry with dissolution, restored into a fresh context, and
both stepped 7 more times: every field bit for bit equal.  The restored
context starts at the other AA parity and with its own compact storage, so
the test also checks that neither enters the arithmetic of a site."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _fields(pkg, lat, cfg):
    out = [lat.field(pkg.FIELD_CONC, s).reshape(-1) for s in range(cfg.n_solutes)]
    out.append(lat.field(pkg.FIELD_BIOMASS, 0).reshape(-1))
    out.append(lat.field(pkg.FIELD_PHASE).reshape(-1))
    out.append(lat.mask().reshape(-1).astype(np.float64))
    return out


def test_checkpoint_restart_is_bit_exact(gpu_lib, pkg, wl):
    mask = wl.sphere_pack(40, 24, 24, 0.45, 2.0, 4.0, seed=91)
    nx, ny, nz = mask.shape
    cfg = wl.coupled_config(pkg, nx, ny, nz, dissolution=True)
    bio = wl.seed_biomass(mask, 92, frac=0.2)
    mineral = wl.seed_mineral(mask, 93, cfg.max_precip_rho)
    a = pkg.Lattice(cfg)
    a.upload_mask(mask)
    a.flow_init()
    a.flow_steps(60)
    a.couple_velocity()
    a.ade_init()
    a.set_field(pkg.FIELD_BIOMASS, 0, bio)
    a.set_field(pkg.FIELD_CONC, 8, mineral)
    for _ in range(5):
        assert a.step(1) == pkg.OK
    nc = cfg.eq.n_comp
    chk = {"flow": a.flow_populations().copy(), "mask": a.mask().copy(),
           "dyn": [a.field(pkg.FIELD_DYNAMICS, k).copy() for k in range(2)],
           "sol": [a.solute_populations(s).copy() for s in range(8)],
           "imm": a.field(pkg.FIELD_CONC, 8).copy(), "bio": a.field(pkg.FIELD_BIOMASS, 0).copy(),
           "phase": a.field(pkg.FIELD_PHASE).copy(),
           "start": [a.field(pkg.FIELD_EQ_START, j).copy() for j in range(2 * nc)]}
    assert np.isfinite(chk["start"][0]).sum() > 0

    b = pkg.Lattice(cfg)
    b.upload_mask(chk["mask"])
    for k in range(2):
        b.set_field(pkg.FIELD_DYNAMICS, k, chk["dyn"][k])
    b.set_flow_populations(chk["flow"])
    b.couple_velocity()
    b.ade_init()
    for s in range(8):
        b.set_solute_populations(s, chk["sol"][s])
    b.set_field(pkg.FIELD_CONC, 8, chk["imm"])
    b.set_field(pkg.FIELD_BIOMASS, 0, chk["bio"])
    b.set_field(pkg.FIELD_PHASE, 0, chk["phase"])
    for j in range(2 * nc):
        b.set_field(pkg.FIELD_EQ_START, j, chk["start"][j])
    # the restored state reads back as it was written
    for s in range(8):
        np.testing.assert_array_equal(b.solute_populations(s), chk["sol"][s])
    for j in range(2 * nc):
        np.testing.assert_array_equal(b.field(pkg.FIELD_EQ_START, j), chk["start"][j])
    for _ in range(7):
        assert a.step(1) == pkg.OK
        assert b.step(1) == pkg.OK
    for k, (fa, fb) in enumerate(zip(_fields(pkg, a, cfg), _fields(pkg, b, cfg))):
        np.testing.assert_array_equal(fa, fb, err_msg="field %d" % k)
    a.close()
    b.close()
