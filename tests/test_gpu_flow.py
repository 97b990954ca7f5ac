"""D3Q19 flow on the GPU (AA pattern, FP32 deviations) against the FP64 oracle.

Tolerances (FP32 populations stored as deviations f - t_i vs FP64):
  velocity and density fields: relative L2 error <= 2e-4 after 300 steps.
  converged iteration count of the ValueTracer loop: within 2 % of the oracle's.
"""
import numpy as np
import pytest

from oracle import oracle as o

pytestmark = pytest.mark.gpu

TOL_FIELD = 2e-4


def rel_l2(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def _pack(wl, nx=22, ny=16, nz=16, por=0.55, seed=7):
    return wl.sphere_pack(nx, ny, nz, por, 2.0, 4.0, seed=seed)


@pytest.mark.parametrize("steps", [1, 2, 7, 300])
def test_flow_steps_match_oracle(gpu_lib, pkg, wl, steps):
    mask = _pack(wl)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(steps)
    ref = o.Flow(cfg, mask)
    ref.step(steps)
    rho_o, u_o = ref.macro()
    u_g = np.stack([lat.field(pkg.FIELD_FLOW_U, k).reshape(-1) for k in range(3)])
    rho_g = lat.field(pkg.FIELD_FLOW_RHO).reshape(-1)
    assert rel_l2(u_g, u_o) < TOL_FIELD
    assert rel_l2(rho_g - 1.0, rho_o - 1.0) < TOL_FIELD
    # populations in natural order, whatever the AA parity
    fg = lat.flow_populations()
    fo = ref.f.reshape(19, -1)
    fluid = np.isin(ref.ns, [2, 3])
    assert rel_l2(fg[:, fluid], fo[:, fluid]) < TOL_FIELD
    lat.close()


def test_flow_nodynamics_touching_pore(gpu_lib, pkg, wl):
    """Solid (NoDynamics) directly against pore, as the shipped example grains
    are: populations stream through the solid, and the GPU must follow."""
    nx, ny, nz = 14, 10, 8
    mask = np.full((nx, ny, nz), 2, np.uint8)
    mask[4:9, 3:7, 2:6] = 0
    mask[:, 0, :] = 1
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.9, rho_in=1.002, rho_out=1.0)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(40)
    ref = o.Flow(cfg, mask)
    ref.step(40)
    _, u_o = ref.macro()
    u_g = np.stack([lat.field(pkg.FIELD_FLOW_U, k).reshape(-1) for k in range(3)])
    assert rel_l2(u_g, u_o) < TOL_FIELD
    lat.close()


def test_flow_solve_converges_like_oracle(gpu_lib, pkg, wl):
    mask = _pack(wl, nx=18, ny=12, nz=12, por=0.6, seed=3)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    it_g, st = lat.flow_solve(20000, 1e-6)
    ref = o.Flow(cfg, mask)
    it_o, _ = ref.solve(20000, 1e-6)
    assert st == pkg.OK
    assert abs(it_g - it_o) <= max(2, 0.02 * it_o), (it_g, it_o)
    _, u_o = ref.macro()
    u_g = np.stack([lat.field(pkg.FIELD_FLOW_U, k).reshape(-1) for k in range(3)])
    assert rel_l2(u_g, u_o) < 1e-3
    lat.close()


def test_poiseuille_gpu(gpu_lib, pkg, wl):
    nx, ny, nz = 24, 18, 4
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.0005, rho_out=1.0)
    lat = pkg.Lattice(cfg)
    lat.upload_mask(wl.channel(nx, ny, nz))
    lat.flow_init()
    # a fixed run to steady state: with FP32 populations the energy tracer's
    # relative spread bottoms out near 1e-8, above a 1e-9 tolerance
    lat.flow_steps(6000)
    ux = lat.field(pkg.FIELD_FLOW_U, 0)[nx // 2, :, 1]
    nu = (0.8 - 0.5) / 3.0
    G = (1.0 / 3.0) * (cfg.rho_in - cfg.rho_out) / (nx - 1)
    y = np.arange(ny)
    ana = G / (2 * nu) * (y - 0.5) * (ny - 1.5 - y)
    err = np.linalg.norm(ux[1:-1] - ana[1:-1]) / np.linalg.norm(ana[1:-1])
    assert err < 0.02
    lat.close()


def test_couple_velocity(gpu_lib, pkg, wl):
    mask = _pack(wl)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, solutes=[{"tau": 0.7}])
    lat = pkg.Lattice(cfg)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(51)
    lat.couple_velocity()
    for k in range(3):
        np.testing.assert_allclose(lat.field(pkg.FIELD_VELOCITY, k), lat.field(pkg.FIELD_FLOW_U, k), rtol=0, atol=0)
    # the coupled field against the FP64 oracle's velocity after the same steps
    fl = o.Flow(cfg, mask)
    fl.step(51)
    _, uo = fl.macro()
    u = np.stack([lat.field(pkg.FIELD_VELOCITY, k).reshape(-1) for k in range(3)])
    assert np.linalg.norm(u - uo) <= 2e-4 * np.linalg.norm(uo)
    lat.close()


def _dilate19(wl, live):
    """live or a D3Q19 neighbour live (x not periodic, y and z periodic)."""
    out = live.copy()
    for (dx, dy, dz) in wl.D3Q19[1:]:
        sh = np.roll(np.roll(live, dy, axis=1), dz, axis=2)
        if dx == 1:
            out[1:] |= sh[:-1]
        elif dx == -1:
            out[:-1] |= sh[1:]
        else:
            out |= sh
    return out


def _sealed_block(wl, nx=22, ny=16, nz=16):
    """A duct with a 7^3 block: a bounce-back shell around a solid (NoDynamics)
    5^3 core that no streaming site reaches."""
    mask = np.full((nx, ny, nz), wl.MAT_PORE, np.uint8)
    mask[8:15, 4:11, 4:11] = wl.MAT_BB
    mask[9:14, 5:10, 5:10] = wl.MAT_SOLID
    return mask


def test_flow_compact_storage_matches_full_layout(gpu_lib, pkg, wl):
    """The compact flow storage (the sites that stream and their D3Q19
    neighbours) against every site stored, which is the full-lattice layout
    (storage index = site index): the same state set in natural order on both,
    then steps of both parities, then the sealed core opened (a mask change
    that stores new sites) and more steps.  Bit-exact: the arithmetic is the
    same, only the addressing differs.  -0.0 marks the unneeded sites of the
    full layout (any nonzero bit pattern is stored; the arithmetic reads it as
    the 0 an unstored site reads as), and compares equal to 0."""
    mask = _sealed_block(wl)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0)
    ns, _ = o.classes(cfg, mask.reshape(-1))
    need = _dilate19(wl, np.isin(ns, [2, 3]).reshape(mask.shape)).reshape(-1)
    assert need.sum() == mask.size - 5 ** 3
    a = pkg.Lattice(cfg)
    a.upload_mask(mask)
    a.flow_init()
    a.flow_steps(41)
    P = a.flow_populations()
    assert np.all(P[:, ~need] == 0.0)
    full = P.copy()
    full[:, ~need] = -0.0
    b = pkg.Lattice(cfg)
    b.upload_mask(mask)
    b.set_flow_populations(full)
    c = pkg.Lattice(cfg)
    c.upload_mask(mask)
    c.set_flow_populations(P)
    np.testing.assert_array_equal(c.flow_populations(), P)
    for lat in (a, b, c):
        lat.flow_steps(7)
    pa, pb, pc = (lat.flow_populations() for lat in (a, b, c))
    np.testing.assert_array_equal(pb, pc)
    np.testing.assert_array_equal(pa, pc)
    # the inner 3^3 of the core reads only core slots at either parity: stored
    # -0.0 on the full layout, unstored 0 on the compact one
    inner = np.zeros(mask.shape, bool)
    inner[10:13, 6:9, 6:9] = True
    inner = inner.reshape(-1)
    assert np.signbit(pb[:, inner]).all() and not np.signbit(pc[:, inner]).any()
    opened = mask.copy()
    opened[8:15, 4:11, 4:11] = wl.MAT_PORE
    for lat in (a, b, c):
        lat.upload_mask(opened)
        lat.flow_steps(9)
    pa, pb, pc = (lat.flow_populations() for lat in (a, b, c))
    np.testing.assert_array_equal(pb, pc)
    np.testing.assert_array_equal(pa, pc)
    core = np.zeros(mask.shape, bool)
    core[9:14, 5:10, 5:10] = True
    assert np.abs(pc[:, core.reshape(-1)]).max() > 0      # the flow reached the opened core
    rho_b, rho_c = b.field(pkg.FIELD_FLOW_RHO), c.field(pkg.FIELD_FLOW_RHO)
    np.testing.assert_array_equal(rho_b, rho_c)
    for lat in (a, b, c):
        lat.close()


def test_flow_populations_need_state(gpu_lib, pkg, wl):
    mask = _sealed_block(wl)
    cfg = pkg.make_config(*mask.shape, tau_ns=0.8)
    lat = pkg.Lattice(cfg)
    with pytest.raises(pkg.CLError):
        lat.flow_populations()                  # no flow field yet
    with pytest.raises(pkg.CLError):
        lat.set_flow_populations(np.zeros((19, mask.size), np.float32))   # no mask yet
    lat.close()


def test_graph_replayed_runs_match_step_by_step(gpu_lib, pkg, wl):
    """Runs of flow steps are replayed from a captured CUDA graph of 32 steps
    (cl_timing on launches them step by step): the same populations bit for
    bit over runs of 70 steps (two graph chunks and six steps), an odd run
    that changes the parity the next capture starts from, a pressure change
    (a new capture), and a converging flow_solve."""
    mask = _pack(wl)
    nx, ny, nz = mask.shape
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0)
    out = []
    for timed in (False, True):
        lat = pkg.Lattice(cfg)
        lat.upload_mask(mask)
        lat.flow_init()
        lat.timing(timed)
        lat.flow_steps(70)
        lat.flow_steps(33)
        lat.flow_steps(64)
        lat.set_flow_pressure(1.002, 1.0)
        lat.flow_steps(70)
        it, _ = lat.flow_solve(20000, 1e-6)
        out.append((lat.flow_populations().copy(), it))
        lat.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    assert out[0][1] == out[1][1]
