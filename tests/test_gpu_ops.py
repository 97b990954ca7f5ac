"""The per-operator entry points (cl_op_*): the transport step taken apart in
the reference's processor order.

  - collide, all reaction operators, stream equals one cl_step to FP32
    rounding (rel. L2 <= 1e-5; the reactions read densities summed after the
    collision instead of before);
  - each operator alone against the FP64 oracle's same processor on the same
    state: collide, then kinetics, then abiotic (surface precipitation), then
    equilibrium, then stream, the fields compared after every call
    (rel. L2 <= 1e-4; the interior between collide and stream, every site
    after stream), and the surrogate operator with the surrogate organisms;
  - calls out of order are refused.
"""
import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _coupled(pkg, wl, seed=81):
    mask = wl.sphere_pack(30, 16, 16, 0.5, 2.0, 3.5, seed=seed)
    nx, ny, nz = mask.shape
    cfg = wl.coupled_config(pkg, nx, ny, nz)
    bio = wl.seed_biomass(mask, seed + 1, frac=0.3)
    return cfg, mask, bio


def _lattice(pkg, cfg, mask, bio, flow=60):
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(flow)
    lat.couple_velocity()
    lat.ade_init()
    for m in range(cfg.n_microbes):
        lat.set_field(pkg.FIELD_BIOMASS, m, bio[m] if bio.ndim == 4 else bio)
    return lat


def test_ops_sequence_equals_step(gpu_lib, pkg, wl):
    cfg, mask, bio = _coupled(pkg, wl)
    a = _lattice(pkg, cfg, mask, bio)
    b = _lattice(pkg, cfg, mask, bio)
    for _ in range(6):
        a.step(1)
        b.op_collide()
        b.op_reactions(pkg.OP_ALL)
        b.op_stream()
    for s in range(cfg.n_solutes):
        assert rel_l2(b.field(pkg.FIELD_CONC, s), a.field(pkg.FIELD_CONC, s)) <= 1e-5, s
    assert rel_l2(b.field(pkg.FIELD_BIOMASS, 0), a.field(pkg.FIELD_BIOMASS, 0)) <= 1e-5
    with pytest.raises(pkg.CLError):
        b.op_stream()                  # stream needs a collide first
    b.op_collide()
    with pytest.raises(pkg.CLError):
        b.step(1)                      # no cl_step inside a taken-apart step
    b.op_stream()
    a.close()
    b.close()


def test_each_operator_against_oracle(gpu_lib, pkg, wl):
    cfg, mask, bio = _coupled(pkg, wl, seed=83)
    lat = _lattice(pkg, cfg, mask, bio)
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)])
    tr = o.Transport(cfg, mask, u=u)
    tr.set_biomass(0, bio)

    # between collide and stream the x boundary planes hold no comparable
    # state: a read there gives the prescribed (Dirichlet) or the adjacent
    # interior (zero-gradient) density, completed on the planes by stream;
    # mid-step the interior is compared, after stream every site
    inner = np.zeros(mask.shape, bool)
    inner[1:-1] = True
    inner = inner.reshape(-1)

    def same(what):
        sel = slice(None) if what == "stream" else inner
        for s in range(cfg.n_solutes):
            g, r = lat.field(pkg.FIELD_CONC, s).reshape(-1)[sel], tr.density(s)[sel]
            e = rel_l2(g, r)
            if not e < 1e-4:
                # where the fields part: the x planes of the largest differences
                full = np.zeros(mask.size)
                full[np.arange(mask.size)[sel]] = np.abs(g - r)
                worst = np.argsort(full)[::-1][:8]
                where = [tuple(int(v) for v in np.unravel_index(w, mask.shape)) for w in worst]
                g, r = lat.field(pkg.FIELD_CONC, s).reshape(-1), tr.density(s)
                pytest.fail("%s: solute %d rel. L2 %.3g; largest at %s (gpu %s, oracle %s)" % (
                    what, s, e, where, g[worst].tolist(), r[worst].tolist()))
        assert rel_l2(lat.field(pkg.FIELD_BIOMASS, 0).reshape(-1), tr.biomass(0)) < 1e-5, what

    for _ in range(3):
        lat.op_collide(); tr.collide(); same("collide")
        lat.op_reactions(pkg.OP_KINETICS); tr.reaction_ops(1); same("kinetics")
        lat.op_reactions(pkg.OP_ABIOTIC); tr.reaction_ops(4); same("abiotic")
        lat.op_reactions(pkg.OP_EQUILIBRIUM); tr.reaction_ops(8); same("equilibrium")
        lat.op_stream(); tr.stream(); same("stream")
    lat.close()


def test_surrogate_operator_against_oracle(gpu_lib, pkg, wl):
    mask = wl.sphere_pack(22, 14, 14, 0.5, 2.0, 3.0, seed=85)
    nx, ny, nz = mask.shape
    cfg = wl.surrogate_config(pkg, nx, ny, nz)
    nets = wl.surrogate_nets(pkg)
    b = np.stack([wl.seed_biomass(mask, 86 + m, frac=0.3, lo=0.005, hi=0.05) for m in range(2)])
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(60)
    lat.couple_velocity()
    for slot in range(2):
        lat.set_surrogate(slot, nets[slot])
    lat.ade_init()
    for m in range(2):
        lat.set_field(pkg.FIELD_BIOMASS, m, b[m])
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, c).reshape(-1) for c in range(3)])
    tr = o.Transport(cfg, mask, u=u)
    tr.set_surrogates(nets)
    for m in range(2):
        tr.set_biomass(m, b[m])
    for _ in range(3):
        lat.op_collide(); tr.collide()
        lat.op_reactions(pkg.OP_SURROGATE); tr.reaction_ops(2)
        lat.op_stream(); tr.stream()
    for s in range(6):
        assert rel_l2(lat.field(pkg.FIELD_CONC, s).reshape(-1), tr.density(s)) < 1e-4, s
    for m in range(2):
        bg, bo = lat.field(pkg.FIELD_BIOMASS, m).reshape(-1), tr.biomass(m)
        assert rel_l2(bg, bo) < 1e-5, m
        assert not np.allclose(bo, b[m].reshape(-1))
    lat.close()
