"""Seeded synthetic inputs with the shapes and value distributions of the five
benchmark workloads (the reference ships no dataset; all inputs are generated).

- sphere_pack: random overlapping spheres until the porosity target, y/z
  periodic; solid voxels linked to a pore voxel by any D3Q19 direction become
  bounce-back (material 1), other solids NoDynamics (material 0), pores 2.  The
  x planes 0 and nx-1 copy planes 1 and nx-2, as readGeometry does
  (src/complab_functions.hh:127-156).
- tableau / speciation_batch: components-and-species systems with integer
  stoichiometry in [-2, 2] and log10 K uniform in [-14, 14], and well-posed
  component totals drawn by sampling the free-component logs first.
- the configuration builders of the 64^3 flow+transport case, the 128^3
  biotic case, and the 256x256x512 coupled case.
"""
import numpy as np

MAT_SOLID, MAT_BB, MAT_PORE, MAT_BIO = 0, 1, 2, 3

D3Q19 = [(0, 0, 0), (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 1, 0), (-1, 0, -1), (-1, 0, 1),
         (0, -1, -1), (0, -1, 1), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1), (1, 0, -1),
         (0, 1, 1), (0, 1, -1)]


def sphere_pack(nx, ny, nz, porosity, rmin, rmax, seed, max_spheres=10_000_000):
    """Material numbers (uint8, shape (nx, ny, nz)).  nx includes the two x
    boundary planes; spheres are placed in the interior planes 1..nx-2."""
    rng = np.random.default_rng(seed)
    nxi = nx - 2
    solid = np.zeros((nxi, ny, nz), bool)
    total = solid.size
    n_solid = 0
    target = (1.0 - porosity) * total
    placed = 0
    while n_solid < target and placed < max_spheres:
        cx, cy, cz = rng.uniform(0, nxi), rng.uniform(0, ny), rng.uniform(0, nz)
        r = rng.uniform(rmin, rmax)
        ir = int(np.ceil(r))
        xs = np.arange(int(np.floor(cx - ir)), int(np.ceil(cx + ir)) + 1)
        xs = xs[(xs >= 0) & (xs < nxi)]
        ys = np.arange(int(np.floor(cy - ir)), int(np.ceil(cy + ir)) + 1)
        zs = np.arange(int(np.floor(cz - ir)), int(np.ceil(cz + ir)) + 1)
        if xs.size == 0:
            placed += 1
            continue
        X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
        inside = (X + 0.5 - cx) ** 2 + (Y + 0.5 - cy) ** 2 + (Z + 0.5 - cz) ** 2 <= r * r
        Xi, Yi, Zi = X[inside], Y[inside] % ny, Z[inside] % nz
        before = solid[Xi, Yi, Zi]
        n_solid += int((~before).sum())
        solid[Xi, Yi, Zi] = True
        placed += 1
    mat = np.full((nx, ny, nz), MAT_PORE, np.uint8)
    mat[1:nx - 1][solid] = MAT_SOLID
    mat[0] = mat[1]
    mat[nx - 1] = mat[nx - 2]
    return mark_bounce_back(mat)


def mark_bounce_back(mat):
    """Solids with a pore/biofilm neighbour along any D3Q19 link become bounce-back."""
    fluid = (mat != MAT_SOLID) & (mat != MAT_BB)
    near = np.zeros_like(fluid)
    nx = mat.shape[0]
    for (dx, dy, dz) in D3Q19[1:]:
        sh = np.roll(np.roll(fluid, dy, axis=1), dz, axis=2)
        if dx == 1:
            near[1:] |= sh[:-1]
        elif dx == -1:
            near[:-1] |= sh[1:]
        else:
            near |= sh
    out = mat.copy()
    out[(mat == MAT_SOLID) & near] = MAT_BB
    return out


def walled_pack(nx, ny, nz, porosity, rmin, rmax, seed):
    """A sphere pack in a duct: bounce-back walls on the four y / z faces, and
    every pore voxel that no face path links to the largest pore cluster made
    solid.  The biofilm automaton moves biomass only across faces and relaxes
    its age field over the reference's distance field, which is zero on the
    last y and z index; a colony in a sealed pore, or on a last-index plane
    whose only inner neighbour is solid, gets an age that never settles, and
    the reference ends its run there.  This geometry has neither."""
    mat = sphere_pack(nx, ny, nz, porosity, rmin, rmax, seed)
    mat[:, 0, :] = mat[:, ny - 1, :] = MAT_BB
    mat[:, :, 0] = mat[:, :, nz - 1] = MAT_BB
    from scipy import ndimage
    pore = (mat != MAT_SOLID) & (mat != MAT_BB)
    lab, n = ndimage.label(pore)          # face connectivity
    if n > 1:
        sizes = np.bincount(lab.reshape(-1))
        sizes[0] = 0
        keep = int(np.argmax(sizes))
        mat[pore & (lab != keep)] = MAT_SOLID
    mat[mat == MAT_BB] = MAT_SOLID
    mat[:, 0, :] = mat[:, ny - 1, :] = MAT_SOLID
    mat[:, :, 0] = mat[:, :, nz - 1] = MAT_SOLID
    return mark_bounce_back(mat)


def channel(nx, ny, nz):
    """Plane channel: walls at y = 0 and y = ny-1 (bounce-back), pore between."""
    mat = np.full((nx, ny, nz), MAT_PORE, np.uint8)
    mat[:, 0, :] = MAT_BB
    mat[:, ny - 1, :] = MAT_BB
    return mat


# ---------------------------------------------------------------- speciation
def tableau(n_comp=5, n_secondary=9, seed=4, stoich_range=2, logk_range=14.0, ph_comp=None):
    """(stoich (ns x nc), logk (ns,), comp_species) with the components first as
    identity rows (logK 0), then secondary species with integer stoichiometry
    and logK ~ U[-logk_range, logk_range].  The pH-like component (the last one
    by default) takes coefficients in [-stoich_range, stoich_range]; the others
    in [0, stoich_range], as in real tableaux where only the proton carries
    negative coefficients.  With negative coefficients on every column almost
    no draw has all component totals positive, which the reference requires
    (totals are floored at 1e-30, part4_eqsolver.hh:535)."""
    rng = np.random.default_rng(seed)
    if ph_comp is None:
        ph_comp = n_comp - 1
    ns = n_comp + n_secondary
    S = np.zeros((ns, n_comp))
    S[:n_comp] = np.eye(n_comp)
    for i in range(n_comp, ns):
        while True:
            row = rng.integers(0, stoich_range + 1, n_comp).astype(float)
            row[ph_comp] = rng.integers(-stoich_range, stoich_range + 1)
            others = np.delete(row, ph_comp)
            if np.count_nonzero(others) >= 1 and np.abs(row).sum() >= 2:
                break
        S[i] = row
    logk = np.zeros(ns)
    logk[n_comp:] = rng.uniform(-logk_range, logk_range, n_secondary)
    return S, logk, list(range(n_comp))


def speciation_batch(S, logk, n, seed, ph_comp=None, tot_lo=1e-6, tot_hi=1e-1, h_lo=1e-9, h_hi=1e-5,
                     max_log_c=0.5):
    """Well-posed batch: sample free-component logs x*, form c* = 10^(logK + S x*)
    and totals T = S^T c*; keep samples with no clamp active (all species in
    [1e-30, 10^max_log_c]) and every total positive, non-pH totals within
    [tot_lo, tot_hi].  Returns (totals (n x nc), x* (n x nc), species c* (n x ns),
    acceptance rate)."""
    rng = np.random.default_rng(seed)
    ns, nc = S.shape
    if ph_comp is None:
        ph_comp = nc - 1
    keep_T, keep_x, keep_c = [], [], []
    got, drawn = 0, 0
    while got < n:
        m = max(4 * (n - got), 4096)
        x = rng.uniform(np.log10(tot_lo) - 1.0, np.log10(tot_hi), (m, nc))
        x[:, ph_comp] = rng.uniform(np.log10(h_lo), np.log10(h_hi), m)
        lc = logk[None, :] + x @ S.T
        ok = (lc <= max_log_c).all(1) & (lc >= -30).all(1)
        c = 10.0 ** np.clip(lc, -30, 1)
        T = c @ S
        ok &= (T > 0).all(1)
        others = [j for j in range(nc) if j != ph_comp]
        ok &= ((T[:, others] >= tot_lo) & (T[:, others] <= tot_hi)).all(1)
        drawn += m
        idx = np.nonzero(ok)[0][: n - got]
        keep_T.append(T[idx]); keep_x.append(x[idx]); keep_c.append(c[idx])
        got += idx.size
        if drawn > 200 * n + 10_000_000:
            raise RuntimeError("tableau gives too few well-posed samples")
    return (np.concatenate(keep_T), np.concatenate(keep_x), np.concatenate(keep_c), got / drawn)


def seed_biomass(mask, seed, frac=0.02, lo=10.0, hi=50.0):
    """Biomass density U[lo, hi] on `frac` of the pore voxels that touch a wall."""
    rng = np.random.default_rng(seed)
    pore = mask == MAT_PORE
    wall = (mask == MAT_SOLID) | (mask == MAT_BB)
    near = np.zeros_like(pore)
    for ax in range(3):
        for sh in (1, -1):
            near |= np.roll(wall, sh, axis=ax)
    cand = pore & near
    cand[0] = False
    cand[-1] = False
    pick = cand & (rng.random(mask.shape) < frac)
    b = np.zeros(mask.shape)
    b[pick] = rng.uniform(lo, hi, int(pick.sum()))
    return b


def biotic_config(pkg, nx, ny, nz, seed=2, bmax=100.0, thrd_frac=0.01, ca_seed=1):
    """Biotic kinetics with the cellular-automaton biofilm: four solutes
    (electron donor, O2, NO3-, product) with D3Q7 tau ~ U[0.6, 0.9]; one
    sessile microbe (material 3) oxidising the donor by O2 or by NO3- with
    dual-Monod rates, Vmax ~ U[1e-5, 1e-4] and Ks ~ U[1e-3, 1e-1] in lattice
    units; the CA redistributes biomass above Bmax (fraction push)."""
    rng = np.random.default_rng(seed)
    taus = rng.uniform(0.6, 0.9, 4)
    inlet = [0.1, 0.05, 0.03, 0.0]
    c0 = [0.05, 0.02, 0.03, 0.0]
    sol = [{"tau": float(taus[s]), "c0": c0[s], "left": "D", "left_value": inlet[s], "right": "N"} for s in range(4)]
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0, solutes=sol, microbes=1,
                          pore_codes=(MAT_PORE,), bio_codes=(MAT_BIO,), dt=1.0)
    cfg.enable_kinetics = 1
    vmax = rng.uniform(1e-5, 1e-4, 2)
    ks = rng.uniform(1e-3, 1e-1, 3)
    pkg.add_rxn(cfg, microbe=0, k=float(vmax[0]), monod=[(0, float(ks[0])), (1, float(ks[1]))],
                nu={0: -1.0, 1: -0.5, 3: 1.0}, yield_=0.3)
    pkg.add_rxn(cfg, microbe=0, k=float(vmax[1]), monod=[(0, float(ks[0])), (2, float(ks[2]))],
                nu={0: -1.0, 2: -0.8, 3: 1.0}, yield_=0.2)
    cfg.decay[0] = 1e-6
    cfg.ca_enabled, cfg.ca_half, cfg.ca_bmax, cfg.ca_thrd_frac = 1, 0, bmax, thrd_frac
    cfg.microbe_code[0] = MAT_BIO
    cfg.ca_seed = ca_seed
    return cfg


# solutes of the coupled workload
COUPLED_SOLUTES = ["DOC", "O2", "NO3-", "HCO3-", "Ca2+", "H+", "CO3--", "CaCO3(aq)", "CaCO3(s)"]


def coupled_config(pkg, nx, ny, nz, seed=5, warm_previous=True, dissolution=False):
    """Flow + 8 mobile solutes + 1 immobile mineral:
      kinetics   dual-Monod oxidation of DOC by O2 and by NO3- (one sessile
                 microbe), Vmax ~ U[1e-5, 1e-4], Ks ~ U[1e-3, 1e-1] per step;
      speciation components CO3--, Ca2+, H+ with HCO3- (= CO3-- + H+, logK
                 10.33) and CaCO3(aq) (= Ca2+ + CO3--, logK 3.2) as secondary
                 species, so every component total is positive at pH 8 (the
                 reference floors totals at 1e-30); Newton to a 1e-10 relative
                 residual every step in every pore voxel, started from the
                 voxel's previous solution (cold start after 4 misses);
      precipitation Ca2+ + CO3-- -> CaCO3(s) on wall-adjacent voxels only,
                 saturation-index driven: rate 1e-6 (Omega - 1) per step above
                 saturation, Omega = [Ca][CO3] / Ksp, log Ksp = -8.48 (calcite);
                 the pore water and the inflow start at the speciated
                 composition of pH 8, free Ca 5e-4 and CO3 2e-5 (Omega ~ 3,
                 precipitating a tenth of the free carbonate per step at a
                 wall); a voxel whose inventory reaches 1.0 becomes solid (node
                 conversion);
      dissolution (with dissolution=True) the sealed voxels carry the CaCO3(s)
                 phase, which acid dissolves at its wetted faces, rate
                 1e-2 [mineral][H+] per step, releasing Ca2+ and HCO3- and
                 consuming H+; a voxel whose mineral falls below 1e-3 of a full
                 voxel reopens (a volume-fraction threshold of ~0; the
                 reference requires a reopen fraction inside (0, 1))."""
    rng = np.random.default_rng(seed)
    taus = rng.uniform(0.6, 0.9, 8)
    # speciated carbonate water: free H+, CO3--, Ca2+ and the complexes they form
    h, co3, ca = 1e-8, 2e-5, 5e-4
    hco3 = 10.0 ** 10.33 * co3 * h
    caco3 = 10.0 ** 3.2 * ca * co3
    inlet = [2e-3, 2.5e-4, 5e-4, hco3, ca, h, co3, caco3]
    c0 = [1e-3, 2.5e-4, 1e-4, hco3, ca, h, co3, caco3]
    sol = [{"tau": float(taus[s]), "c0": c0[s], "left": "D", "left_value": inlet[s], "right": "N"} for s in range(8)]
    sol.append({"immobile": True, "c0": 0.0})
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.0005, rho_out=1.0, solutes=sol, microbes=1, dt=1.0)
    vmax = rng.uniform(1e-5, 1e-4, 2)
    ks = rng.uniform(1e-3, 1e-1, 3)
    cfg.enable_kinetics = 1
    pkg.add_rxn(cfg, microbe=0, k=float(vmax[0]), monod=[(0, float(ks[0])), (1, float(ks[1]))],
                nu={0: -1.0, 1: -1.0, 3: 1.0}, yield_=0.3)
    pkg.add_rxn(cfg, microbe=0, k=float(vmax[1]), monod=[(0, float(ks[0])), (2, float(ks[2]))],
                nu={0: -1.0, 2: -0.8, 3: 1.0}, yield_=0.2)
    cfg.decay[0] = 1e-7
    cfg.enable_abiotic = 1
    cfg.precip_enabled = 1
    cfg.abiotic_surface_only = 1
    cfg.precip_substrate = 8
    cfg.max_precip_rho = 1.0
    cfg.precip_code = MAT_SOLID
    pkg.add_rxn(cfg, k=1e-6, mass=[4, 6], nu={4: -1.0, 6: -1.0, 8: 1.0}, ksp=10.0 ** -8.48)
    cfg.use_equilibrium = 1
    S = np.zeros((9, 3))
    S[6, 0] = 1; S[4, 1] = 1; S[5, 2] = 1
    S[3] = [1, 0, 1]
    S[7] = [1, 1, 0]
    logk = [0, 0, 0, 10.33, 0, 0, 0, 3.2, 0]
    pkg.set_eq_system(cfg.eq, S, logk, [6, 4, 5], max_iter=100, tol=1e-10, warm_iter=4)
    cfg.eq_warm_previous = 1 if warm_previous else 0
    if dissolution:
        cfg.dissol_enabled = 1
        cfg.reopen_fraction = 1e-3
        cfg.dissol_surface_only = 1
        cfg.dissol_apply_at_walls = 1
        pkg.add_phase(cfg, substrate=8, full_density=cfg.max_precip_rho, is_precipitate=True,
                      k=1e-2, mass=[5], nu={4: 1.0, 3: 1.0, 5: -1.0})
    return cfg


def seed_mineral(mask, seed, full, frac=0.5):
    """Pre-existing mineral coatings: an inventory U[0, full) on `frac` of the
    wall-adjacent pore voxels of x = 1..nx-2, so that precipitation carries some
    of them across the conversion threshold during a run."""
    rng = np.random.default_rng(seed)
    pore = mask == MAT_PORE
    wall = (mask == MAT_SOLID) | (mask == MAT_BB)
    near = np.zeros_like(pore)
    for ax in range(3):
        for sh in (1, -1):
            near |= np.roll(wall, sh, axis=ax)
    cand = pore & near
    cand[0] = False
    cand[-1] = False
    pick = cand & (rng.random(mask.shape) < frac)
    m = np.zeros(mask.shape)
    m[pick] = rng.uniform(0.0, full, int(pick.sum()))
    return m


def cold_species(S, T, comp_species=None):
    """Species vector a voxel would hold before equilibration: each component's
    own species at its total (the reference's cold start reads these), every
    other species at the floor."""
    n = T.shape[0]
    ns, nc = S.shape
    c = np.full((n, ns), 1e-30)
    cs = comp_species if comp_species is not None else list(range(nc))
    for j in range(nc):
        if cs[j] >= 0:
            c[:, cs[j]] = T[:, j]
    return c


def surrogate_nets(pkg, seed=0):
    """Two organism networks, 3 -> 20 tanh -> 20 tanh -> 4 linear, weights
    ~N(0, 0.3); inputs (donor, acceptor, biomass) clamped to their mapminmax
    box; outputs (growth 1/h, donor uptake, acceptor uptake, product uptake),
    uptakes in mmol/gDW/h (positive = consumed, so the product's is negative)."""
    rng = np.random.default_rng(seed)
    nets = []
    for o in range(2):
        widths = [3, 20, 20, 4]
        W = [rng.normal(0, 0.3, (widths[l + 1], widths[l])) for l in range(3)]
        b = [rng.normal(0, 0.3, widths[l + 1]) for l in range(3)]
        lo = np.array([0.0, 0.0, 0.0])
        hi = np.array([2e-3, 1e-3, 60.0])
        gain = 2.0 / (hi - lo)
        # output box: growth 0..0.4 1/h, uptakes 0..8, product -8..0
        y_lo = np.array([0.0, 0.0, 0.0, -8.0])
        y_hi = np.array([0.4, 8.0, 8.0, 0.0])
        nets.append(pkg.make_surrogate_net(widths, W, b, lo, gain, y_lo, 2.0 / (y_hi - y_lo), x_lo=lo, x_hi=hi))
    return nets


def surrogate_config(pkg, nx, ny, nz, seed=6):
    """Six solutes (donor, acceptor, product of each of two organisms) fed by
    the surrogate reaction type of two organisms on sessile biomass."""
    rng = np.random.default_rng(seed)
    taus = rng.uniform(0.6, 0.9, 6)
    inlet = [1e-3, 5e-4, 0.0, 1e-3, 5e-4, 0.0]
    sol = [{"tau": float(taus[s]), "c0": inlet[s] * 0.5, "left": "D", "left_value": inlet[s], "right": "N"}
           for s in range(6)]
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.0005, rho_out=1.0, solutes=sol, microbes=2, dt=360.0)
    cfg.n_srg = 2
    for o in range(2):
        g = cfg.srg[o]
        g.microbe, g.net = o, o
        base = 3 * o
        for i, (kind, idx) in enumerate([(pkg.SRG_IN_CONC, base), (pkg.SRG_IN_CONC, base + 1),
                                         (pkg.SRG_IN_BIOMASS, 0)]):
            g.in_kind[i], g.in_index[i] = kind, idx
        for q, (kind, idx) in enumerate([(pkg.SRG_OUT_GROWTH, 0), (pkg.SRG_OUT_FOUT, base),
                                         (pkg.SRG_OUT_FOUT, base + 1), (pkg.SRG_OUT_FOUT, base + 2)]):
            g.out_kind[q], g.out_index[q] = kind, idx
        for s in range(6):
            g.kc[s] = 1e-4
            g.vmax[s] = 5.0 if s in (base, base + 1) else 0.0
        g.mw = 24.6
        g.kd = 1e-7
    return cfg
