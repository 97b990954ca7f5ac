"""Python mirror of the CompLB3D hot-path operator surface over libcomplab_gpu.so.

The reference drives its hot path through Palabos data processors
(``applyProcessingFunctional(new run_kinetics(...), box, lattices)``,
src/complab.cpp:1152-1860).  Here the same operators are methods of
:class:`Lattice`, each one a call into the C ABI declared in
include/complab_gpu.h; the arithmetic runs in the hand-written sm_100a
kernels of csrc/.  There is no CPU fallback: importing this module without the
built library, or calling it without a GPU, raises.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcomplab_gpu.so")

MAX_SOLUTES, MAX_MICROBES, MAX_RXN, MAX_MONOD = 32, 12, 16, 3
MAX_COMP, MAX_SPECIES, MAX_CODES, MAX_PHASES = 24, 128, 8, 4
SRG_MAX_LAYERS, SRG_MAX_WIDTH = 5, 32

OK, WARN_NOT_CONVERGED = 0, 1
ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_DIVERGED = -1, -2, -3, -4, -5
BC_DIRICHLET, BC_NEUMANN = 0, 1
FIELD_CONC, FIELD_BIOMASS, FIELD_VELOCITY, FIELD_FLOW_RHO, FIELD_FLOW_U, FIELD_PHASE, FIELD_EQ_ITERS = range(7)
FIELD_CA_AGE, FIELD_CA_TOTAL, FIELD_EQ_START, FIELD_DYNAMICS = 7, 8, 9, 10
RED_SUM, RED_MIN, RED_MAX, RED_COUNT_EQ = range(4)
EQ_START_COLD, EQ_START_GIVEN, EQ_START_LEARNED = range(3)
EQ_NET_TCGEN05, EQ_NET_MMA_SYNC = 0, 1
EQ_SOLVER_NEWTON, EQ_SOLVER_PCF = 0, 1
SRG_TENSOR, SRG_FP32, SRG_TCGEN05 = 0, 1, 2
MAX_SRG_ORG = 2
SRG_IN_FIN, SRG_IN_CONC, SRG_IN_BIOMASS = 0, 1, 2
SRG_OUT_GROWTH, SRG_OUT_FOUT = 0, 1
KERNEL_ADE_MAIN, KERNEL_FLOW_STEP, KERNEL_ADE_REACT = 0, 1, 2
OPT_COMPILED_CHEM, OPT_FAST_VARIANT, OPT_EQ_LEARN, OPT_EQ_FORGET, OPT_EQ_LEARN_TRAININGS = 1, 2, 3, 4, 5
CHEM_COUPLED, CHEM_BIOTIC4, CHEM_ZHAO24, CHEM_SURROGATE2 = 1, 2, 3, 4
OP_KINETICS, OP_SURROGATE, OP_ABIOTIC, OP_EQUILIBRIUM, OP_ALL = 1, 2, 4, 8, 15
RATELAW_TABLE, RATELAW_ZHAO = 0, 1

c_int32, c_double, c_int64 = ctypes.c_int32, ctypes.c_double, ctypes.c_int64


class Rxn(ctypes.Structure):
    _fields_ = [("microbe", c_int32), ("n_monod", c_int32), ("monod_s", c_int32 * MAX_MONOD),
                ("monod_ks", c_double * MAX_MONOD), ("n_mass", c_int32), ("mass_s", c_int32 * 2),
                ("k", c_double), ("nu", c_double * MAX_SOLUTES), ("yield_", c_double), ("ksp", c_double)]


class EqSystem(ctypes.Structure):
    _fields_ = [("n_comp", c_int32), ("n_species", c_int32), ("comp_species", c_int32 * MAX_COMP),
                ("stoich", (c_double * MAX_COMP) * MAX_SPECIES), ("logk", c_double * MAX_SPECIES),
                ("max_iter", c_int32), ("tol", c_double), ("warm_iter", c_int32),
                ("solver", c_int32), ("anderson_depth", c_int32)]


class Phase(ctypes.Structure):
    _fields_ = [("id", c_int32), ("material", c_int32), ("substrate", c_int32), ("is_precipitate", c_int32),
                ("full_density", c_double), ("initial_fill", c_double), ("k", c_double), ("n_mass", c_int32),
                ("mass_s", c_int32 * 2), ("nu", c_double * MAX_SOLUTES)]


class SurrogateNet(ctypes.Structure):
    _fields_ = [("n_layers", c_int32), ("widths", c_int32 * (SRG_MAX_LAYERS + 1)),
                ("x_offset", c_double * SRG_MAX_WIDTH), ("x_gain", c_double * SRG_MAX_WIDTH), ("x_ymin", c_double),
                ("y_offset", c_double * SRG_MAX_WIDTH), ("y_gain", c_double * SRG_MAX_WIDTH), ("y_ymin", c_double),
                ("x_lo", c_double * SRG_MAX_WIDTH), ("x_hi", c_double * SRG_MAX_WIDTH),
                ("params", c_double * 4096)]


class SrgOrganism(ctypes.Structure):
    _fields_ = [("microbe", c_int32), ("net", c_int32),
                ("in_kind", c_int32 * SRG_MAX_WIDTH), ("in_index", c_int32 * SRG_MAX_WIDTH),
                ("out_kind", c_int32 * SRG_MAX_WIDTH), ("out_index", c_int32 * SRG_MAX_WIDTH),
                ("kc", c_double * MAX_SOLUTES), ("vmax", c_double * MAX_SOLUTES), ("mw", c_double), ("kd", c_double)]


class Config(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32), ("nz", c_int32),
        ("solid_code", c_int32), ("bb_code", c_int32),
        ("n_pore_codes", c_int32), ("pore_codes", c_int32 * MAX_CODES),
        ("n_bio_codes", c_int32), ("bio_codes", c_int32 * MAX_CODES),
        ("tau_ns", c_double), ("perm_ratio", c_double), ("rho_in", c_double), ("rho_out", c_double),
        ("n_solutes", c_int32),
        ("omega_pore", c_double * MAX_SOLUTES), ("omega_bio", c_double * MAX_SOLUTES),
        ("immobile", c_int32 * MAX_SOLUTES),
        ("left_type", c_int32 * MAX_SOLUTES), ("right_type", c_int32 * MAX_SOLUTES),
        ("left_value", c_double * MAX_SOLUTES), ("right_value", c_double * MAX_SOLUTES),
        ("c0", c_double * MAX_SOLUTES),
        ("n_microbes", c_int32), ("b_max", c_double), ("thrd_bfilm_frac", c_double), ("dt", c_double),
        ("enable_kinetics", c_int32), ("enable_abiotic", c_int32), ("abiotic_surface_only", c_int32),
        ("n_rxn", c_int32), ("rxn", Rxn * MAX_RXN), ("decay", c_double * MAX_MICROBES),
        ("use_equilibrium", c_int32), ("eq", EqSystem), ("eq_warm_previous", c_int32),
        ("precip_enabled", c_int32), ("precip_substrate", c_int32), ("max_precip_rho", c_double),
        ("precip_code", c_int32), ("precip_phase_id", c_int32),
        ("dissol_enabled", c_int32), ("reopen_fraction", c_double), ("dissol_surface_only", c_int32),
        ("dissol_apply_at_walls", c_int32),
        ("n_phases", c_int32), ("phases", Phase * MAX_PHASES),
        ("n_srg", c_int32), ("srg", SrgOrganism * MAX_SRG_ORG),
        ("ca_enabled", c_int32), ("ca_half", c_int32), ("ca_bmax", c_double), ("ca_thrd_frac", c_double),
        ("microbe_code", c_int32 * MAX_MICROBES), ("ca_seed", ctypes.c_uint64),
        ("rate_law", c_int32), ("microbe_carrier", c_int32 * MAX_MICROBES),
    ]


_lib = None


def load_library(path=LIB_PATH):
    """Load the CUDA library; raises if it was not built (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libcomplab_gpu.so is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    vp, P = ctypes.c_void_p, ctypes.POINTER
    lib.cl_create.restype = vp
    lib.cl_create.argtypes = [P(Config), vp, P(ctypes.c_int)]
    lib.cl_last_error.restype = ctypes.c_char_p
    for name, args in [
        ("cl_destroy", [vp]), ("cl_upload_mask", [vp, vp]), ("cl_download_mask", [vp, vp]),
        ("cl_flow_init", [vp]), ("cl_flow_steps", [vp, c_int32]),
        ("cl_flow_solve", [vp, c_int32, c_double, P(c_int32)]), ("cl_flow_energy", [vp, P(c_double)]),
        ("cl_couple_velocity", [vp]), ("cl_update_dynamics", [vp]), ("cl_ade_init", [vp]),
        ("cl_step", [vp, c_int32]), ("cl_get_field", [vp, c_int32, c_int32, vp]),
        ("cl_set_field", [vp, c_int32, c_int32, vp]), ("cl_get_flow_populations", [vp, vp]),
        ("cl_set_flow_populations", [vp, vp]), ("cl_get_solute_populations", [vp, c_int32, vp]),
        ("cl_set_solute_populations", [vp, c_int32, vp]),
        ("cl_reduce", [vp, c_int32, c_int32, c_int32, c_double, P(c_double)]),
        ("cl_precip_convert", [vp, P(c_int64)]), ("cl_dissol_convert", [vp, P(c_int64)]),
        ("cl_flow_velocity_stats", [vp, P(c_double), P(c_double), P(c_double)]),
        ("cl_flow_velocity_norm_masked", [vp, c_int32, P(c_double), P(c_int64)]),
        ("cl_set_option", [vp, c_int32, c_int64]), ("cl_get_option", [vp, c_int32, P(c_int64)]),
        ("cl_op_collide", [vp]), ("cl_op_stream", [vp]), ("cl_op_reactions", [vp, c_int32]),
        ("cl_op_kinetics", [vp]), ("cl_op_surrogate", [vp]), ("cl_op_abiotic", [vp]), ("cl_op_equilibrium", [vp]),
        ("cl_set_flow_pressure", [vp, c_double, c_double]), ("cl_set_transport", [vp, vp, vp, c_double]),
        ("cl_device_bytes", [vp, P(ctypes.c_uint64)]), ("cl_abi_sizes", [vp, c_int32]),
        ("cl_timing_enable", [vp, c_int32]), ("cl_timing_read", [vp, c_int32, P(c_double), P(c_int64)]),
        ("cl_launch_count", [vp, P(c_int64)]), ("cl_set_surrogate", [vp, c_int32, vp]),
        ("cl_ca_redistribute", [vp, P(c_int32), P(c_int64), P(c_double)]), ("cl_ca_update_mask", [vp, P(c_int64)]), ("cl_fd_diffuse", [vp, c_double, ctypes.c_uint32]),
        ("cl_math_exp10", [vp, vp, c_int64, c_int32]),
    ]:
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = args
    _lib = lib
    return lib


def math_exp10(x, which=0):
    """The library's FP64 10^x (which=0, the Newton solves' own) or CUDA's
    exp10 (which=1) on the GPU, for accuracy checks."""
    lib = load_library()
    xs = np.ascontiguousarray(x, np.float64)
    y = np.zeros_like(xs)
    _check(lib, lib.cl_math_exp10(_ptr(xs), _ptr(y), xs.size, which), "cl_math_exp10")
    return y


def check_abi(lib=None):
    """Compare ctypes struct sizes with the library's sizeof values."""
    lib = lib or load_library()
    sizes = (c_int32 * 5)()
    n = lib.cl_abi_sizes(sizes, 5)
    want = [ctypes.sizeof(Config), ctypes.sizeof(Rxn), ctypes.sizeof(EqSystem),
            ctypes.sizeof(Phase), ctypes.sizeof(SurrogateNet)]
    got = list(sizes)[:n]
    if got != want:
        raise RuntimeError("ABI mismatch: library %s, binding %s" % (got, want))
    return got


class CLError(RuntimeError):
    pass


def _check(lib, st, what):
    if st < 0:
        raise CLError("%s failed (%d): %s" % (what, st, lib.cl_last_error().decode()))
    return st


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def omega_from_tau(tau):
    return 1.0 / tau


def make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0, solutes=(), microbes=0,
                solid_code=0, bb_code=1, pore_codes=(2,), bio_codes=(), perm_ratio=0.0, dt=1.0):
    """Build a Config.  ``solutes`` is a list of dicts with keys tau (or
    tau_bio), c0, left/right ('D' Dirichlet or 'N' zero-gradient), left_value,
    right_value, immobile."""
    c = Config()
    c.nx, c.ny, c.nz = nx, ny, nz
    c.solid_code, c.bb_code = solid_code, bb_code
    c.n_pore_codes = len(pore_codes)
    for i, v in enumerate(pore_codes):
        c.pore_codes[i] = v
    c.n_bio_codes = len(bio_codes)
    for i, v in enumerate(bio_codes):
        c.bio_codes[i] = v
    c.tau_ns, c.perm_ratio, c.rho_in, c.rho_out = tau_ns, perm_ratio, rho_in, rho_out
    c.n_solutes = len(solutes)
    for s, d in enumerate(solutes):
        tau = d.get("tau", 0.8)
        c.omega_pore[s] = 1.0 / tau
        c.omega_bio[s] = 1.0 / d.get("tau_bio", tau)
        c.immobile[s] = 1 if d.get("immobile") else 0
        c.left_type[s] = BC_NEUMANN if d.get("left", "N") == "N" else BC_DIRICHLET
        c.right_type[s] = BC_NEUMANN if d.get("right", "N") == "N" else BC_DIRICHLET
        c.left_value[s] = d.get("left_value", 0.0)
        c.right_value[s] = d.get("right_value", 0.0)
        c.c0[s] = d.get("c0", 0.0)
    c.n_microbes = microbes
    c.dt = dt
    c.eq.max_iter, c.eq.tol, c.eq.warm_iter = 100, 1e-10, 8
    return c


def add_rxn(cfg, microbe=-1, k=0.0, monod=(), mass=(), nu=None, yield_=0.0, ksp=0.0):
    """Append one table-driven rate expression to cfg (ksp > 0: the
    mass-action product P enters as max(P / ksp - 1, 0))."""
    r = cfg.rxn[cfg.n_rxn]
    r.microbe, r.k, r.yield_, r.ksp = microbe, k, yield_, ksp
    r.n_monod = len(monod)
    for j, (s, ks) in enumerate(monod):
        r.monod_s[j], r.monod_ks[j] = s, ks
    r.n_mass = len(mass)
    for j, s in enumerate(mass):
        r.mass_s[j] = s
    for s, v in (nu or {}).items():
        r.nu[s] = v
    cfg.n_rxn += 1
    return r


def add_phase(cfg, substrate, full_density, material=0, initial_fill=0.0, is_precipitate=False,
              k=0.0, mass=(), nu=None):
    """Append one dissolvable phase (id = its position + 1) with its rate law
    rate = k * mineral * prod water[mass]; products nu[s] * rate.  A phase
    marked is_precipitate becomes the one precipitation stamps."""
    ph = cfg.phases[cfg.n_phases]
    ph.id = cfg.n_phases + 1
    ph.material, ph.substrate, ph.is_precipitate = material, substrate, 1 if is_precipitate else 0
    ph.full_density, ph.initial_fill, ph.k = full_density, initial_fill, k
    ph.n_mass = len(mass)
    for j, sidx in enumerate(mass):
        ph.mass_s[j] = sidx
    for sidx, v in (nu or {}).items():
        ph.nu[sidx] = v
    cfg.n_phases += 1
    if is_precipitate:
        cfg.precip_phase_id = ph.id
    return ph


def set_eq_system(sys, stoich, logk, comp_species, max_iter=100, tol=1e-10, warm_iter=8, solver=0,
                  anderson_depth=0):
    """Fill an EqSystem from an (ns x nc) stoichiometry matrix.  solver:
    EQ_SOLVER_NEWTON or EQ_SOLVER_PCF (the reference's live PCF + Anderson)."""
    stoich = np.asarray(stoich, float)
    ns, nc = stoich.shape
    sys.n_comp, sys.n_species = nc, ns
    for j in range(MAX_COMP):
        sys.comp_species[j] = comp_species[j] if j < nc else -1
    for i in range(ns):
        for j in range(nc):
            sys.stoich[i][j] = stoich[i, j]
        sys.logk[i] = logk[i]
    sys.max_iter, sys.tol, sys.warm_iter = max_iter, tol, warm_iter
    sys.solver, sys.anderson_depth = solver, anderson_depth
    return sys


class Lattice:
    """One device context: the flow lattice, the solute lattices and the
    per-voxel fields, stepped in the reference's operator order."""

    def __init__(self, cfg, stream=None):
        self.lib = load_library()
        self.cfg = cfg
        self.N = cfg.nx * cfg.ny * cfg.nz
        self.shape = (cfg.nx, cfg.ny, cfg.nz)
        st = ctypes.c_int(0)
        self.h = self.lib.cl_create(ctypes.byref(cfg), ctypes.c_void_p(stream) if stream else None, ctypes.byref(st))
        if not self.h:
            raise CLError("cl_create failed (%d): %s" % (st.value, self.lib.cl_last_error().decode()))

    def close(self):
        if self.h:
            self.lib.cl_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _c(self, st, what):
        return _check(self.lib, st, what)

    # geometry
    def upload_mask(self, mask):
        m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
        assert m.size == self.N
        self._c(self.lib.cl_upload_mask(self.h, _ptr(m)), "cl_upload_mask")

    def mask(self):
        m = np.empty(self.N, np.uint8)
        self._c(self.lib.cl_download_mask(self.h, _ptr(m)), "cl_download_mask")
        return m.reshape(self.shape)

    # flow
    def flow_init(self):
        self._c(self.lib.cl_flow_init(self.h), "cl_flow_init")

    def flow_steps(self, n):
        self._c(self.lib.cl_flow_steps(self.h, n), "cl_flow_steps")

    def flow_solve(self, max_it, eps):
        it = c_int32(0)
        st = self._c(self.lib.cl_flow_solve(self.h, max_it, eps, ctypes.byref(it)), "cl_flow_solve")
        return it.value, st

    def flow_energy(self):
        e = c_double(0)
        self._c(self.lib.cl_flow_energy(self.h, ctypes.byref(e)), "cl_flow_energy")
        return e.value

    def couple_velocity(self):
        self._c(self.lib.cl_couple_velocity(self.h), "cl_couple_velocity")

    def update_dynamics(self):
        self._c(self.lib.cl_update_dynamics(self.h), "cl_update_dynamics")

    # transport
    def ade_init(self):
        self._c(self.lib.cl_ade_init(self.h), "cl_ade_init")

    def step(self, n=1):
        return self._c(self.lib.cl_step(self.h, n), "cl_step")

    # the step taken apart (the reference's processor calls)
    def op_collide(self):
        return self._c(self.lib.cl_op_collide(self.h), "cl_op_collide")

    def op_reactions(self, ops=OP_ALL):
        return self._c(self.lib.cl_op_reactions(self.h, ops), "cl_op_reactions")

    def op_stream(self):
        return self._c(self.lib.cl_op_stream(self.h), "cl_op_stream")

    def set_option(self, key, value):
        self._c(self.lib.cl_set_option(self.h, key, int(value)), "cl_set_option")

    def get_option(self, key):
        v = c_int64(0)
        self._c(self.lib.cl_get_option(self.h, key, ctypes.byref(v)), "cl_get_option")
        return v.value

    def field(self, field, index=0):
        out = np.empty(self.N, np.float64)
        self._c(self.lib.cl_get_field(self.h, field, index, _ptr(out)), "cl_get_field")
        return out.reshape(self.shape)

    def set_field(self, field, index, values):
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        assert v.size == self.N
        self._c(self.lib.cl_set_field(self.h, field, index, _ptr(v)), "cl_set_field")

    def flow_populations(self):
        out = np.empty(19 * self.N, np.float32)
        self._c(self.lib.cl_get_flow_populations(self.h, _ptr(out)), "cl_get_flow_populations")
        return out.reshape(19, self.N)

    def set_flow_populations(self, f):
        v = np.ascontiguousarray(f, dtype=np.float32).reshape(-1)
        self._c(self.lib.cl_set_flow_populations(self.h, _ptr(v)), "cl_set_flow_populations")

    def solute_populations(self, s):
        out = np.empty(7 * self.N, np.float32)
        self._c(self.lib.cl_get_solute_populations(self.h, s, _ptr(out)), "cl_get_solute_populations")
        return out.reshape(7, self.N)

    def set_solute_populations(self, s, g):
        v = np.ascontiguousarray(g, dtype=np.float32).reshape(-1)
        assert v.size == 7 * self.N
        self._c(self.lib.cl_set_solute_populations(self.h, s, _ptr(v)), "cl_set_solute_populations")

    def reduce(self, field, index, op, arg=0.0):
        out = c_double(0)
        self._c(self.lib.cl_reduce(self.h, field, index, op, arg, ctypes.byref(out)), "cl_reduce")
        return out.value

    def precip_convert(self):
        ch = c_int64(0)
        self._c(self.lib.cl_precip_convert(self.h, ctypes.byref(ch)), "cl_precip_convert")
        return ch.value

    def velocity_stats(self):
        """(mean |u| and max u_x over x = 1..nx-2, mean u_x at x = nx-2)."""
        a, b, c = c_double(), c_double(), c_double()
        self._c(self.lib.cl_flow_velocity_stats(self.h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
                "cl_flow_velocity_stats")
        return a.value, b.value, c.value

    def velocity_norm_masked(self, code):
        """(sum of |u|, site count) over the sites of material `code` in x = 1..nx-2."""
        a, n = c_double(), c_int64()
        self._c(self.lib.cl_flow_velocity_norm_masked(self.h, code, ctypes.byref(a), ctypes.byref(n)),
                "cl_flow_velocity_norm_masked")
        return a.value, n.value

    def set_flow_pressure(self, rho_in, rho_out):
        self._c(self.lib.cl_set_flow_pressure(self.h, rho_in, rho_out), "cl_set_flow_pressure")

    def set_transport(self, omega_pore, omega_bio, dt):
        op = np.ascontiguousarray(omega_pore, np.float64)
        ob = np.ascontiguousarray(omega_bio, np.float64)
        self._c(self.lib.cl_set_transport(self.h, _ptr(op), _ptr(ob), dt), "cl_set_transport")

    def dissol_convert(self):
        ch = c_int64(0)
        self._c(self.lib.cl_dissol_convert(self.h, ctypes.byref(ch)), "cl_dissol_convert")
        return ch.value

    def ca_update_mask(self):
        """Initial mask update after seeding the biomass; returns sites changed."""
        ch = c_int64(0)
        self._c(self.lib.cl_ca_update_mask(self.h, ctypes.byref(ch)), "cl_ca_update_mask")
        return ch.value

    def fd_diffuse(self, nu, microbes):
        """One finite-difference step of the sessile biomass of the microbes whose bit is set."""
        self._c(self.lib.cl_fd_diffuse(self.h, float(nu), int(microbes)), "cl_fd_diffuse")

    def ca_redistribute(self):
        """One CA block: returns (status, push sweeps, sites whose mask changed, biomass maximum)."""
        sw, ch, bm = c_int32(0), c_int64(0), c_double(0)
        st = self._c(self.lib.cl_ca_redistribute(self.h, ctypes.byref(sw), ctypes.byref(ch), ctypes.byref(bm)),
                     "cl_ca_redistribute")
        return st, sw.value, ch.value, bm.value

    def timing(self, on=True):
        self._c(self.lib.cl_timing_enable(self.h, 1 if on else 0), "cl_timing_enable")

    def timing_read(self, kernel):
        ms, n = c_double(0), c_int64(0)
        self._c(self.lib.cl_timing_read(self.h, kernel, ctypes.byref(ms), ctypes.byref(n)), "cl_timing_read")
        return ms.value, n.value

    def launch_count(self):
        n = c_int64(0)
        self._c(self.lib.cl_launch_count(self.h, ctypes.byref(n)), "cl_launch_count")
        return n.value

    def set_surrogate(self, slot, net):
        self._c(self.lib.cl_set_surrogate(self.h, slot, ctypes.byref(net)), "cl_set_surrogate")

    def device_bytes(self):
        b = ctypes.c_uint64(0)
        self._c(self.lib.cl_device_bytes(self.h, ctypes.byref(b)), "cl_device_bytes")
        return b.value


# ---------------------------------------------------------------- speciation
def _bind_eq(lib):
    if getattr(lib, "_eq_bound", False):
        return
    vp, P = ctypes.c_void_p, ctypes.POINTER
    lib.cl_eq_create.restype = vp
    lib.cl_eq_create.argtypes = [P(EqSystem), vp, P(ctypes.c_int)]
    for name, args in [
        ("cl_eq_destroy", [vp]),
        ("cl_eq_solve_device", [vp, vp, vp, vp, vp, vp, c_int64, c_int32]),
        ("cl_eq_solve_host", [vp, vp, vp, vp, vp, vp, c_int64, c_int32]),
        ("cl_eq_train", [vp, vp, vp, c_int64, c_int32, c_int32, ctypes.c_float, ctypes.c_uint64,
                         P(ctypes.c_float)]),
        ("cl_eq_grad_host", [vp, vp, vp, c_int32, P(ctypes.c_float), vp]),
        ("cl_eq_param_count", [vp, P(c_int32)]), ("cl_eq_get_params", [vp, vp]),
        ("cl_eq_set_params", [vp, vp]), ("cl_eq_predict_host", [vp, vp, vp, c_int32]), ("cl_eq_set_network_path", [vp, c_int32]),
        ("cl_eq_predict_device", [vp, vp, vp, c_int64]),
        ("cl_eq_pcf_device", [vp, vp, vp, vp, vp, c_int64]), ("cl_eq_pcf_host", [vp, vp, vp, vp, vp, c_int64]),
        ("cl_surrogate_batch_device", [P(SurrogateNet), vp, vp, c_int64, c_int32, vp]),
        ("cl_surrogate_batch_host", [P(SurrogateNet), vp, vp, c_int64, c_int32]),
    ]:
        fn = getattr(lib, name)
        fn.restype = ctypes.c_int
        fn.argtypes = args
    lib._eq_bound = True


class EqSolver:
    """Batched FP64 Newton speciation with a learned warm start.  Mirrors the
    reference's EquilibriumChemistry::calculate_species_concentrations
    (src/complab3d_processors_part4_eqsolver.hh:1187-1214) for a whole batch."""

    def __init__(self, sys, stream=None):
        self.lib = load_library()
        _bind_eq(self.lib)
        self.sys = sys
        self.nc, self.ns = sys.n_comp, sys.n_species
        st = ctypes.c_int(0)
        self.h = self.lib.cl_eq_create(ctypes.byref(sys), ctypes.c_void_p(stream) if stream else None,
                                       ctypes.byref(st))
        if not self.h:
            raise CLError("cl_eq_create failed (%d): %s" % (st.value, self.lib.cl_last_error().decode()))
        n = c_int32(0)
        self.lib.cl_eq_param_count(self.h, ctypes.byref(n))
        self.n_params = n.value

    def close(self):
        if self.h:
            self.lib.cl_eq_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, totals, cold_species=None, x0=None, start=EQ_START_COLD):
        T = np.ascontiguousarray(totals, np.float64)
        n = T.shape[0]
        x = np.zeros((n, self.nc)) if x0 is None else np.array(x0, np.float64, copy=True)
        it = np.zeros(n, np.int32)
        stt = np.zeros(n, np.uint8)
        cs = None if cold_species is None else np.ascontiguousarray(cold_species, np.float64)
        _check(self.lib, self.lib.cl_eq_solve_host(self.h, _ptr(T), _ptr(cs) if cs is not None else None, _ptr(x),
                                                   _ptr(it), _ptr(stt), n, start), "cl_eq_solve_host")
        return x, it, stt

    def pcf(self, species):
        """The reference's live solve (PCF + Anderson) of each row of species
        (n x n_species): species out, iterations, converged flags."""
        c = np.ascontiguousarray(species, np.float64).reshape(-1, self.ns)
        n = c.shape[0]
        out = np.zeros_like(c)
        it = np.zeros(n, np.int32)
        cv = np.zeros(n, np.uint8)
        _check(self.lib, self.lib.cl_eq_pcf_host(self.h, _ptr(c), _ptr(out), _ptr(it), _ptr(cv), n), "cl_eq_pcf_host")
        return out, it, cv

    def pcf_device(self, d_in, d_out, d_iters, d_conv, n):
        """PCF + Anderson on device species rows (device pointers)."""
        return _check(self.lib, self.lib.cl_eq_pcf_device(self.h, d_in, d_out, d_iters, d_conv, n),
                      "cl_eq_pcf_device")

    def solve_device(self, d_totals, d_cold, d_x, d_iters, d_status, n, start):
        """Device-pointer variant (ints from torch.Tensor.data_ptr())."""
        return _check(self.lib, self.lib.cl_eq_solve_device(self.h, d_totals, d_cold, d_x, d_iters, d_status, n,
                                                            start), "cl_eq_solve_device")

    def predict_device(self, d_totals, d_x, n):
        """The network's Newton start for n device totals (device pointers)."""
        return _check(self.lib, self.lib.cl_eq_predict_device(self.h, d_totals, d_x, n), "cl_eq_predict_device")

    def train_device(self, d_totals, d_logfree, n, epochs=10, batch=1024, lr=2e-3, seed=0):
        loss = ctypes.c_float(0)
        _check(self.lib, self.lib.cl_eq_train(self.h, d_totals, d_logfree, n, epochs, batch, lr, seed,
                                              ctypes.byref(loss)), "cl_eq_train")
        return loss.value

    def grad(self, x, y):
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_float(0)
        _check(self.lib, self.lib.cl_eq_grad_host(self.h, _ptr(x), _ptr(y), x.shape[0], ctypes.byref(loss),
                                                  _ptr(g)), "cl_eq_grad_host")
        return loss.value, g

    def params(self):
        p = np.zeros(self.n_params, np.float32)
        _check(self.lib, self.lib.cl_eq_get_params(self.h, _ptr(p)), "cl_eq_get_params")
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        _check(self.lib, self.lib.cl_eq_set_params(self.h, _ptr(p)), "cl_eq_set_params")

    def set_network_path(self, path):
        """EQ_NET_TCGEN05 (default) or EQ_NET_MMA_SYNC for the network's inference."""
        _check(self.lib, self.lib.cl_eq_set_network_path(self.h, path), "cl_eq_set_network_path")

    def predict(self, x):
        x = np.ascontiguousarray(x, np.float32)
        y = np.zeros_like(x)
        _check(self.lib, self.lib.cl_eq_predict_host(self.h, _ptr(x), _ptr(y), x.shape[0]), "cl_eq_predict_host")
        return y


def make_surrogate_net(widths, weights, biases, x_offset, x_gain, y_offset, y_gain, x_lo=None, x_hi=None,
                       x_ymin=-1.0, y_ymin=-1.0):
    """Pack a feed-forward network (weights[l] of shape (out, in)) with its
    mapminmax settings into a SurrogateNet."""
    net = SurrogateNet()
    net.n_layers = len(widths) - 1
    for l, w in enumerate(widths):
        net.widths[l] = w
    flat = []
    for W, b in zip(weights, biases):
        flat.extend(np.asarray(W, np.float64).reshape(-1).tolist())
        flat.extend(np.asarray(b, np.float64).reshape(-1).tolist())
    for i, v in enumerate(flat):
        net.params[i] = v
    for i in range(widths[0]):
        net.x_offset[i], net.x_gain[i] = x_offset[i], x_gain[i]
        net.x_lo[i] = -1e300 if x_lo is None else x_lo[i]
        net.x_hi[i] = 1e300 if x_hi is None else x_hi[i]
    for o in range(widths[-1]):
        net.y_offset[o], net.y_gain[o] = y_offset[o], y_gain[o]
    net.x_ymin, net.y_ymin = x_ymin, y_ymin
    return net


def surrogate_batch(net, x, mode=SRG_TENSOR):
    lib = load_library()
    _bind_eq(lib)
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros((x.shape[0], net.widths[net.n_layers]), np.float32)
    _check(lib, lib.cl_surrogate_batch_host(ctypes.byref(net), _ptr(x), _ptr(y), x.shape[0], mode),
           "cl_surrogate_batch_host")
    return y


def surrogate_batch_device(net, d_x, d_y, n, mode=SRG_TENSOR, stream=None):
    lib = load_library()
    _bind_eq(lib)
    return _check(lib, lib.cl_surrogate_batch_device(ctypes.byref(net), d_x, d_y, n, mode, stream),
                  "cl_surrogate_batch_device")
