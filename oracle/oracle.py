"""ctypes binding of the FP64 CPU oracle (liboracle.so) and of the reference's
own Palabos-free code compiled from its sources (_ref/libref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by the CPU legs of bench.py, always as the checker or the timed CPU baseline,
never as the product path.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")

_orc = None
_ref = None


def build():
    """Compile liboracle.so (and _ref/libref.so when the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True, stdout=sys.stderr)


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def lib():
    global _orc
    if _orc is None:
        # make is a no-op when liboracle.so is newer than its sources and the
        # public header whose structs it reads
        build()
        _orc = ctypes.CDLL(LIB)
        vp, d, i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int
        _orc.orc_flow_step.restype = d
        _orc.orc_flow_step.argtypes = [vp, vp, vp, vp]
        _orc.orc_flow_solve.restype = i
        _orc.orc_flow_solve.argtypes = [vp, vp, vp, vp, i, d, vp]
        _orc.orc_transport_step.restype = ctypes.c_int64
        _orc.orc_transport_step.argtypes = [vp, vp]
        _orc.orc_reaction_stage.restype = ctypes.c_int64
        _orc.orc_reaction_stage.argtypes = [vp, vp]
        _orc.orc_reaction_ops.restype = ctypes.c_int64
        _orc.orc_reaction_ops.argtypes = [vp, vp, i]
        _orc.orc_collide.restype = None
        _orc.orc_collide.argtypes = [vp, vp]
        _orc.orc_stream.restype = None
        _orc.orc_stream.argtypes = [vp, vp]
        _orc.orc_precip_convert.restype = ctypes.c_int64
        _orc.orc_precip_convert.argtypes = [vp, vp]
        _orc.orc_dissol_convert.restype = ctypes.c_int64
        _orc.orc_dissol_convert.argtypes = [vp, vp]
        _orc.orc_eq_newton.restype = i
        _orc.orc_eq_newton.argtypes = [vp, vp, vp, i, d, vp]
        _orc.orc_eq_residual.restype = d
        _orc.orc_eq_residual.argtypes = [vp, vp, vp]
        _orc.orc_eq_batch.restype = None
        _orc.orc_eq_batch.argtypes = [vp, vp, vp, vp, vp, vp, ctypes.c_int64, i]
        _orc.orc_pcf_batch.restype = None
        _orc.orc_pcf_batch.argtypes = [vp, vp, vp, vp, vp, ctypes.c_int64]
        _orc.orc_mlp_forward_backward.restype = d
        _orc.orc_mlp_forward_backward.argtypes = [i, i, i, vp, vp, vp, i, vp, vp]
        _orc.orc_surrogate_forward.restype = None
        _orc.orc_surrogate_forward.argtypes = [vp, vp, vp, ctypes.c_int64]
        _orc.orc_rates.restype = None
        _orc.orc_rates.argtypes = [vp, i, vp, vp, vp, vp]
        _orc.orc_ca_init.restype = None
        _orc.orc_ca_init.argtypes = [vp, vp, vp]
        _orc.orc_ca_update_mask.restype = ctypes.c_int64
        _orc.orc_ca_update_mask.argtypes = [vp, vp, vp, i]
        _orc.orc_ca_redistribute.restype = i
        _orc.orc_ca_redistribute.argtypes = [vp, vp, vp, i, vp, vp, vp]
        _orc.orc_fd_diffuse.restype = None
        _orc.orc_fd_diffuse.argtypes = [vp, vp, d, ctypes.c_uint32]
    return _orc


def ref_lib():
    """The reference's own code; None when it was not built (no reference tree)."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        _ref = ctypes.CDLL(REF_LIB)
    return _ref


class OrcState(ctypes.Structure):
    _fields_ = [("g", ctypes.c_void_p), ("g_tmp", ctypes.c_void_p), ("imm", ctypes.c_void_p),
                ("bio", ctypes.c_void_p), ("u", ctypes.c_void_p), ("mask", ctypes.c_void_p),
                ("ade_class", ctypes.c_void_p), ("rho_bc", ctypes.c_void_p), ("eq_iters", ctypes.c_void_p),
                ("srg_nets", ctypes.c_void_p), ("phase", ctypes.c_void_p),
                ("kin", ctypes.c_void_p), ("abio", ctypes.c_void_p)]


class OrcCa(ctypes.Structure):
    _fields_ = [("total", ctypes.c_void_p), ("age", ctypes.c_void_p), ("distpos", ctypes.c_void_p),
                ("out", ctypes.c_void_p), ("sweeps", ctypes.c_uint64), ("mask_sum", ctypes.c_int64),
                ("draws", ctypes.c_uint64)]


def check_config_layout(cfg):
    """The oracle reads cl_config through the public header: its sizeof must
    match the ctypes mirror, or every field after the change is misread."""
    got = lib().orc_config_size()
    if got != ctypes.sizeof(cfg):
        raise RuntimeError("liboracle.so was built against another cl_config (%d vs %d bytes): rebuild it"
                           % (got, ctypes.sizeof(cfg)))


def classes(cfg, mask):
    N = mask.size
    ns = np.empty(N, np.uint8)
    ad = np.empty(N, np.uint8)
    lib().orc_classes_from_mask(ctypes.byref(cfg), _p(np.ascontiguousarray(mask, np.uint8).reshape(-1)), _p(ns), _p(ad))
    return ns, ad


class Flow:
    """FP64 flow lattice (deviation populations, natural order)."""

    def __init__(self, cfg, mask):
        check_config_layout(cfg)
        self.cfg = cfg
        self.N = cfg.nx * cfg.ny * cfg.nz
        self.mask = np.ascontiguousarray(mask, np.uint8).reshape(-1)
        self.ns, self.ade = classes(cfg, self.mask)
        self.f = np.zeros(19 * self.N)
        self.tmp = np.zeros(19 * self.N)
        lib().orc_flow_init(ctypes.byref(cfg), _p(self.ns), _p(self.f))

    def step(self, n=1):
        e = 0.0
        for _ in range(n):
            e = lib().orc_flow_step(ctypes.byref(self.cfg), _p(self.ns), _p(self.f), _p(self.tmp))
            self.f, self.tmp = self.tmp, self.f
        return e

    def solve(self, max_it, eps):
        hist = np.zeros(max(max_it, 1))
        it = lib().orc_flow_solve(ctypes.byref(self.cfg), _p(self.ns), _p(self.f), _p(self.tmp), max_it, eps, _p(hist))
        return it, hist

    def macro(self):
        rho = np.zeros(self.N)
        u = np.zeros(3 * self.N)
        lib().orc_flow_macro(ctypes.byref(self.cfg), _p(self.ns), _p(self.f), _p(rho), _p(u))
        return rho, u.reshape(3, self.N)


class Transport:
    """FP64 solute lattices stepped in the reference's processor order."""

    def __init__(self, cfg, mask, u=None):
        check_config_layout(cfg)
        self.cfg = cfg
        N = self.N = cfg.nx * cfg.ny * cfg.nz
        S, M = cfg.n_solutes, max(cfg.n_microbes, 1)
        self.mask = np.ascontiguousarray(mask, np.uint8).reshape(-1).copy()
        self.ns, self.ade = classes(cfg, self.mask)
        self.g = np.zeros(S * 7 * N)
        self.g_tmp = np.zeros(S * 7 * N)
        self.imm = np.zeros(S * N)
        self.bio = np.zeros(M * N)
        self.u = np.zeros(3 * N) if u is None else np.ascontiguousarray(u, np.float64).reshape(-1).copy()
        self.rho_bc = np.zeros(S * 2 * cfg.ny * cfg.nz)
        self.eq_iters = np.zeros(N, np.int32)
        self.phase = np.zeros(N, np.uint8)
        self.st = OrcState(_p(self.g).value, _p(self.g_tmp).value, _p(self.imm).value, _p(self.bio).value,
                           _p(self.u).value, _p(self.mask).value, _p(self.ade).value, _p(self.rho_bc).value,
                           _p(self.eq_iters).value, None, _p(self.phase).value)
        self._nets = None
        lib().orc_ade_init(ctypes.byref(cfg), ctypes.byref(self.st))

    def step(self, n=1):
        nc = 0
        for _ in range(n):
            nc += lib().orc_transport_step(ctypes.byref(self.cfg), ctypes.byref(self.st))
        return nc

    def density(self, s):
        out = np.zeros(self.N)
        lib().orc_solute_density(ctypes.byref(self.cfg), ctypes.byref(self.st), s, _p(out))
        return out

    def set_conc(self, s, values):
        v = np.asarray(values, np.float64).reshape(-1)
        if self.cfg.immobile[s]:
            self.imm[s * self.N:(s + 1) * self.N] = v
        else:
            t = np.array([0.25] + [0.125] * 6)
            for i in range(7):
                self.g[(s * 7 + i) * self.N:(s * 7 + i + 1) * self.N] = t[i] * v

    def set_surrogates(self, nets):
        """Networks of the surrogate organisms (a sequence of SurrogateNet, one per slot)."""
        arr = (type(nets[0]) * len(nets))(*nets)
        self._nets = arr
        self.st.srg_nets = ctypes.addressof(arr)

    def set_rate_law(self, kin_addr, abio_addr):
        """Compiled rate laws (C function addresses with the signatures of
        orc_state.kin / orc_state.abio) in place of the rate table."""
        self.st.kin = kin_addr
        self.st.abio = abio_addr

    def set_biomass(self, m, values):
        self.bio[m * self.N:(m + 1) * self.N] = np.asarray(values, np.float64).reshape(-1)

    def biomass(self, m):
        return self.bio[m * self.N:(m + 1) * self.N].copy()

    def precip_convert(self):
        return lib().orc_precip_convert(ctypes.byref(self.cfg), ctypes.byref(self.st))

    def collide(self):
        lib().orc_collide(ctypes.byref(self.cfg), ctypes.byref(self.st))

    def reaction_ops(self, ops):
        """The reaction processors selected by ops (1 kinetics, 2 surrogate,
        4 abiotic + dissolution, 8 equilibrium) on the current state."""
        return lib().orc_reaction_ops(ctypes.byref(self.cfg), ctypes.byref(self.st), ops)

    def stream(self):
        lib().orc_stream(ctypes.byref(self.cfg), ctypes.byref(self.st))

    def reaction_stage(self):
        """The reaction stage of a step alone (no collide, no stream)."""
        return lib().orc_reaction_stage(ctypes.byref(self.cfg), ctypes.byref(self.st))

    def dissol_convert(self):
        return lib().orc_dissol_convert(ctypes.byref(self.cfg), ctypes.byref(self.st))

    # cellular-automaton biofilm
    def ca_init(self):
        N, M = self.N, max(self.cfg.n_microbes, 1)
        self.ca_total = np.zeros(N)
        self.ca_age = np.zeros(N, np.int32)
        self.ca_distpos = np.zeros(N, np.uint8)
        self.ca_out = np.zeros(6 * M * N)
        self.ca = OrcCa(_p(self.ca_total).value, _p(self.ca_age).value, _p(self.ca_distpos).value,
                        _p(self.ca_out).value, 0, 0, 0)
        lib().orc_ca_init(ctypes.byref(self.cfg), _p(self.mask), ctypes.byref(self.ca))

    def ca_update_mask(self, serial=False):
        return lib().orc_ca_update_mask(ctypes.byref(self.cfg), ctypes.byref(self.st), ctypes.byref(self.ca),
                                        1 if serial else 0)

    def fd_diffuse(self, nu, microbes):
        """fdDiffusion3D of the sessile biomass of the microbes whose bit is set."""
        lib().orc_fd_diffuse(ctypes.byref(self.cfg), ctypes.byref(self.st), float(nu), int(microbes))

    def ca_redistribute(self, serial=False):
        """(status, sweeps, mask changes, biomass maximum) of one CA block."""
        sw, ch, bm = ctypes.c_int32(0), ctypes.c_int64(0), ctypes.c_double(0)
        st = lib().orc_ca_redistribute(ctypes.byref(self.cfg), ctypes.byref(self.st), ctypes.byref(self.ca),
                                       1 if serial else 0, ctypes.byref(sw), ctypes.byref(ch), ctypes.byref(bm))
        return st, sw.value, ch.value, bm.value


def eq_batch(sys, totals, cold_species, x0=None, start=0):
    n = totals.shape[0]
    nc = sys.n_comp
    x = np.zeros((n, nc)) if x0 is None else np.array(x0, np.float64, copy=True)
    it = np.zeros(n, np.int32)
    stt = np.zeros(n, np.uint8)
    lib().orc_eq_batch(ctypes.byref(sys), _p(np.ascontiguousarray(totals, np.float64)),
                       _p(np.ascontiguousarray(cold_species, np.float64)), _p(x), _p(it), _p(stt),
                       ctypes.c_int64(n), start)
    return x, it, stt


def pcf_batch(sys, species):
    """The reference's live solve (PCF + Anderson) of each row of species:
    (species out, iterations, converged)."""
    c = np.ascontiguousarray(species, np.float64).reshape(-1, sys.n_species)
    n = c.shape[0]
    out = np.zeros_like(c)
    it = np.zeros(n, np.int32)
    cv = np.zeros(n, np.uint8)
    lib().orc_pcf_batch(ctypes.byref(sys), _p(c), _p(out), _p(it), _p(cv), ctypes.c_int64(n))
    return out, it, cv


def eq_residual(sys, totals, x):
    t = np.ascontiguousarray(totals, np.float64)
    xx = np.ascontiguousarray(x, np.float64)
    return np.array([lib().orc_eq_residual(ctypes.byref(sys), _p(t[k]), _p(xx[k])) for k in range(t.shape[0])])


def mlp_forward_backward(n_in, H, n_out, params, x, y, want_grad=True):
    p = np.ascontiguousarray(params, np.float64)
    x = np.ascontiguousarray(x, np.float64)
    y = np.ascontiguousarray(y, np.float64)
    g = np.zeros_like(p) if want_grad else None
    yh = np.zeros((x.shape[0], n_out))
    loss = lib().orc_mlp_forward_backward(n_in, H, n_out, _p(p), _p(x), _p(y), x.shape[0], _p(g), _p(yh))
    return loss, g, yh


def surrogate_forward(net, x):
    x = np.ascontiguousarray(x, np.float64)
    n = x.shape[0]
    y = np.zeros((n, net.widths[net.n_layers]))
    lib().orc_surrogate_forward(ctypes.byref(net), _p(x), _p(y), ctypes.c_int64(n))
    return y


def rates(cfg, abiotic, C, B=None):
    S, M = cfg.n_solutes, max(cfg.n_microbes, 1)
    R = np.zeros(S)
    BR = np.zeros(M)
    Bv = np.zeros(M) if B is None else np.asarray(B, np.float64)
    lib().orc_rates(ctypes.byref(cfg), abiotic, _p(np.asarray(C, np.float64)), _p(Bv), _p(R), _p(BR))
    return R, BR


# ---- reference's own code -------------------------------------------------
def ref_pcf_solve(stoich, logk, comp_species, species, max_iter=200, tol=1e-10, depth=4):
    r = ref_lib()
    stoich = np.ascontiguousarray(stoich, np.float64)
    ns, nc = stoich.shape
    species = np.ascontiguousarray(species, np.float64).reshape(-1, ns)
    n = species.shape[0]
    out = np.zeros_like(species)
    it = np.zeros(n, np.int32)
    cv = np.zeros(n, np.uint8)
    cs = np.ascontiguousarray(comp_species, np.int32)
    r.ref_pcf_solve(nc, ns, _p(stoich), _p(np.ascontiguousarray(logk, np.float64)), _p(cs), _p(species),
                    _p(out), _p(it), _p(cv), ctypes.c_int64(n), max_iter, ctypes.c_double(tol), depth)
    return out, it, cv


def ref_surrogate(fin):
    fin = np.ascontiguousarray(fin, np.float64).reshape(-1, 2)
    out = np.zeros(fin.shape[0])
    ref_lib().ref_surrogate(_p(fin), _p(out), ctypes.c_int64(fin.shape[0]))
    return out


def ref_kinetics_ex05(B, C, mask=2):
    B = np.asarray(B, np.float64); C = np.asarray(C, np.float64)
    sr = np.zeros(C.size); br = np.zeros(B.size)
    ref_lib().ref_kinetics_ex05(_p(B), B.size, _p(C), C.size, mask, _p(sr), _p(br))
    return sr, br


def ref_abiotic_ex13(C, mask=2):
    C = np.asarray(C, np.float64)
    sr = np.zeros(C.size)
    ref_lib().ref_abiotic_ex13(_p(C), C.size, mask, _p(sr))
    return sr


class RefCa:
    """The reference's own CA processors on one block (oracle/ref/ca_harness.cpp),
    carrying the same state as Transport's CA arrays: mask, biomass, total,
    age, the distance sign, the draw counter and the mask-sum baseline."""

    def __init__(self, cfg, mask, bio, distpos, total=None, age=None, mask_sum=None):
        lib_ = ref_lib()
        if lib_ is None:
            raise RuntimeError("oracle/_ref/libref.so is not built")
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        lib_.ref_ca_block.restype = i
        lib_.ref_ca_block.argtypes = [i, i, i, i, i, d, d, i, i, vp, i, vp, ctypes.c_uint64, vp,
                                      vp, vp, vp, vp, vp, vp, vp, vp, vp]
        lib_.ref_ca_update_mask.restype = ctypes.c_longlong
        lib_.ref_ca_update_mask.argtypes = [i, i, i, i, i, d, d, i, i, vp, i, vp, vp, vp, vp, vp, vp, vp]
        self.lib, self.cfg = lib_, cfg
        N = cfg.nx * cfg.ny * cfg.nz
        M = cfg.n_microbes
        self.mask = np.ascontiguousarray(mask, np.uint8).reshape(-1).copy()
        self.bio = np.ascontiguousarray(bio, np.float64).reshape(-1)[:M * N].copy()
        self.total = np.zeros(N) if total is None else np.array(total, np.float64).reshape(-1)
        self.age = np.array(age, np.int32).reshape(-1) if age is not None else None
        self.distpos = np.ascontiguousarray(distpos, np.uint8).reshape(-1).copy()
        self.pore = np.array(list(cfg.pore_codes)[:cfg.n_pore_codes], np.int32)
        self.codes = np.array(list(cfg.microbe_code)[:M], np.int32)
        self.draws = ctypes.c_uint64(0)
        self.mask_sum = ctypes.c_longlong(int(self.mask.astype(np.int64).sum()) if mask_sum is None else mask_sum)

    def _head(self):
        c = self.cfg
        return (c.nx, c.ny, c.nz, c.n_microbes, c.ca_half, c.ca_bmax, c.ca_thrd_frac, c.solid_code, c.bb_code,
                _p(self.pore), int(self.pore.size), _p(self.codes))

    def update_mask(self):
        return self.lib.ref_ca_update_mask(*self._head(), _p(self.mask), _p(self.bio), _p(self.total),
                                           _p(self.age), _p(self.distpos), ctypes.byref(self.mask_sum))

    def block(self):
        sw, ch, gm = ctypes.c_int32(0), ctypes.c_longlong(0), ctypes.c_double(0)
        st = self.lib.ref_ca_block(*self._head(), self.cfg.ca_seed, ctypes.byref(self.draws), _p(self.mask),
                                   _p(self.bio), _p(self.total), _p(self.age), _p(self.distpos),
                                   ctypes.byref(self.mask_sum), ctypes.byref(sw), ctypes.byref(ch), ctypes.byref(gm))
        return st, sw.value, gm.value


_rxn = {}


def rxn_lib(variant):
    """The reference's reaction processors on one block (oracle/ref/rxn_harness.cpp):
    variant 13 binds the rate laws of examples 05 + 13, variant 14 those of 05 + 14.
    None when the reference tree was absent at build time."""
    if variant not in _rxn:
        path = os.path.join(HERE, "_ref", "librxn%d.so" % variant)
        if not os.path.exists(path):
            return None
        L = ctypes.CDLL(path)
        vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
        L.ref_rxn_stage.restype = i
        L.ref_rxn_stage.argtypes = [i, i, i, i, i, d, i, i, i, vp, vp, vp, vp,
                                    i, vp, vp, vp, vp, vp, d, i, vp, i,
                                    i, vp, vp, vp, i, d, i]
        L.ref_precip_convert.restype = ctypes.c_longlong
        L.ref_precip_convert.argtypes = [i, i, i, vp, d, i, i, i, i, vp, vp]
        L.ref_dissol_convert.restype = ctypes.c_longlong
        L.ref_dissol_convert.argtypes = [i, i, i, i, vp, i, i, i, i, vp, vp, vp, vp, vp, d, vp, vp]
        _rxn[variant] = L
    return _rxn[variant]


RXN_KINETICS, RXN_ABIOTIC, RXN_SURFACE, RXN_DISSOLUTION, RXN_EQUILIBRIUM = 1, 2, 4, 8, 16


def _phase_arrays(cfg):
    n = cfg.n_phases
    ids = np.array([cfg.phases[k].id for k in range(n)] or [0], np.int32)
    mat = np.array([cfg.phases[k].material for k in range(n)] or [0], np.int32)
    sub = np.array([cfg.phases[k].substrate for k in range(n)] or [0], np.int32)
    full = np.array([cfg.phases[k].full_density for k in range(n)] or [0.0])
    prec = np.array([cfg.phases[k].is_precipitate for k in range(n)] or [0], np.int32)
    return n, ids, mat, sub, full, prec


def ref_rxn_stage(variant, cfg, mask, phase, C, B, flags, eq_depth=4):
    """Run the reference's reaction stage on densities C (S x N) and biomass
    B (M x N); returns the new (C, B)."""
    L = rxn_lib(variant)
    N = cfg.nx * cfg.ny * cfg.nz
    S, M = cfg.n_solutes, cfg.n_microbes
    C = np.array(C, np.float64).reshape(S, N).copy()
    B = np.array(B, np.float64).reshape(max(M, 1), N)[:max(M, 1)].copy()
    mask = np.ascontiguousarray(mask, np.uint8).reshape(-1)
    phase = np.ascontiguousarray(phase if phase is not None else np.zeros(N), np.uint8).reshape(-1)
    n, ids, mat, sub, full, prec = _phase_arrays(cfg)
    pore = np.array(list(cfg.pore_codes)[:cfg.n_pore_codes], np.int32)
    e = cfg.eq
    nc = e.n_comp
    stoich = np.array([[e.stoich[i][j] for j in range(nc)] for i in range(S)] if nc else [[0.0]], np.float64)
    logk = np.array([e.logk[i] for i in range(S)], np.float64)
    cs = np.array([e.comp_species[j] for j in range(max(nc, 1))], np.int32)
    L.ref_rxn_stage(cfg.nx, cfg.ny, cfg.nz, S, M, cfg.dt, cfg.solid_code, cfg.bb_code, flags,
                    _p(mask), _p(phase), _p(C), _p(B), n, _p(ids), _p(mat), _p(sub), _p(full), _p(prec),
                    cfg.reopen_fraction, cfg.dissol_surface_only, _p(pore), int(pore.size),
                    nc, _p(stoich), _p(logk), _p(cs), e.max_iter, e.tol, eq_depth)
    return C, B


def ref_precip_convert(cfg, P, mask, phase):
    L = rxn_lib(13)
    mask = np.ascontiguousarray(mask, np.uint8).reshape(-1).copy()
    phase = np.ascontiguousarray(phase, np.uint8).reshape(-1).copy()
    P = np.ascontiguousarray(P, np.float64).reshape(-1)
    ch = L.ref_precip_convert(cfg.nx, cfg.ny, cfg.nz, _p(P), cfg.max_precip_rho, cfg.solid_code, cfg.bb_code,
                              cfg.precip_code, cfg.precip_phase_id, _p(mask), _p(phase))
    return ch, mask, phase


def ref_dissol_convert(cfg, C, mask, phase):
    L = rxn_lib(14)
    mask = np.ascontiguousarray(mask, np.uint8).reshape(-1).copy()
    phase = np.ascontiguousarray(phase, np.uint8).reshape(-1).copy()
    C = np.ascontiguousarray(C, np.float64).reshape(-1)
    n, ids, mat, sub, full, prec = _phase_arrays(cfg)
    pore0 = cfg.pore_codes[0] if cfg.n_pore_codes else 2
    ch = L.ref_dissol_convert(cfg.nx, cfg.ny, cfg.nz, cfg.n_solutes, _p(C), pore0, cfg.solid_code, cfg.bb_code,
                              n, _p(ids), _p(mat), _p(sub), _p(full), _p(prec), cfg.reopen_fraction,
                              _p(mask), _p(phase))
    return ch, mask, phase
