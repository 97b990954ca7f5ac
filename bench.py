#!/usr/bin/env python
"""Benchmark of the CompLB3D hot path on B200.

Headline: coupled-step MLUPS of the 256x256x512 sphere-pack workload (porosity
0.35): one transport step (D3Q7 ADR of 8 mobile solutes with dual-Monod
kinetics, surface-gated CaCO3 precipitation and a 3-component Newton
speciation in every pore voxel: a reaction launch over the reactive sites and
a streaming launch, slab by slab) plus the amortised flow re-solve (500 D3Q19
steps every 200 transport steps = 2.5 flow steps per step) and the node
conversion every 200 steps.  Inputs are resident in HBM; the state (~13 GB) is
far larger than L2, so no flush is needed between steps.

The same line reports the learned-vs-cold Newton speciation batch (2^21
solves of a 5-component x 14-species tableau at a 1e-10 relative residual,
network trained on 2^20 Newton-produced pairs), the roofline of the transport
step (its reaction and streaming launches, timed together with CUDA events on
the context's stream), the biotic + CA workload, an end-to-end figure through the
C ABI with host buffers, and the FP64 CPU oracle timed on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
Under torchrun each rank runs its own domain (weak scaling, no collective on
the data path); the timed region is bracketed by a barrier and the max over
ranks is reported.
"""
import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "complb3d-lattice-boltzmann-fba-surrogate-cobrapy-glpk_b200")
METRIC = "coupled-step MLUPS on 1 B200; learned vs cold Newton speciation at 1e-10 residual"
FULL = (512, 256, 256)          # nx (flow direction, incl. the two boundary planes), ny, nz
CPU_SAMPLE = (128, 64, 64)      # bounded sample of the same workload for the CPU legs
ADE_BYTES_PER_FLUID_SITE = 8 * 56 + 12 + 8 + 8   # 8 solutes x (7 f32 read + write), u, mineral, biomass
FLOW_BYTES_PER_BGK_SITE = 19 * 4 * 2


def load_pkg():
    if "complab_b200" in sys.modules:
        return sys.modules["complab_b200"]
    spec = importlib.util.spec_from_file_location("complab_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["complab_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_workloads():
    load_pkg()
    import importlib
    return importlib.import_module("complab_b200.workloads")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(kernel):
    """DRAM bytes per fluid site from the committed ncu summary, or None."""
    p = os.path.join(ROOT, "profiles", "ade_step_coupled_traffic.txt")
    if not os.path.exists(p):
        return None
    for line in open(p):
        parts = line.split()
        if len(parts) >= 2 and parts[0] == kernel:
            return float(parts[1])
    return None


class Clocks:
    """SM clock and clock-event reasons sampled during the timed region: an
    NVML thread every 10 ms (plus one sample at start and one at stop, so a
    short region still has some), or nvidia-smi at 200 ms without NVML."""
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.nv = None
        self.p = None
        self.sm, self.reasons, self.mx = [], set(), None
        try:
            import pynvml as nv
            nv.nvmlInit()
            try:
                import torch
                uuid = str(torch.cuda.get_device_properties(dev).uuid)
                h = nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
            except Exception:
                h = nv.nvmlDeviceGetHandleByIndex(dev)
            self.mx = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                         "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                         "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                         "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            self.nv, self.h = nv, h
        except Exception:
            self.nv = None
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)

    def _sample(self):
        nv = self.nv
        self.sm.append(float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)))
        r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
        for k, b in self.bits.items():
            if r & b:
                self.reasons.add(k)

    def _loop(self):
        while not self.stop_ev.wait(0.01):
            self._sample()

    def start(self):
        if self.nv is not None:
            import threading
            self._sample()
            self.stop_ev = threading.Event()
            self.th = threading.Thread(target=self._loop, daemon=True)
            self.th.start()
            return
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.nv is not None:
            self._sample()
            self.stop_ev.set()
            self.th.join()
            return {"sm_mhz": statistics.median(self.sm), "sm_max_mhz": self.mx, "reasons": sorted(self.reasons),
                    "samples": len(self.sm), "source": "nvml"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.strip().split(",") for l in open(self.f.name) if l.strip()]
        sm, mx, reasons = [], None, set()
        for r in rows:
            r = [x.strip() for x in r]
            try:
                sm.append(float(r[1])); mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(self.NAMES):
                if len(r) > 5 + k and r[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi"}


def max_over_ranks(value, dist=None, device=None):
    """Max of a per-rank duration over the process group (identity alone)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_mlups(sites_per_rank, world, steps, ms):
    """Whole-job throughput: every rank advances its own domain (weak scaling)."""
    return sites_per_rank * world * steps / (ms * 1e-3) / 1e6


def coupled_setup(pkg, wl, shape, seed, stream=None):
    """The coupled workload: sphere pack, the coupled chemistry with
    saturation-driven precipitation and acid dissolution of the precipitate,
    biomass on 2% of the wall-adjacent pore voxels, and mineral coatings
    U[0, 1) of a full voxel on half of them (so node conversions happen)."""
    nx, ny, nz = shape
    mask = wl.sphere_pack(nx, ny, nz, 0.35, 5.0, 10.0, seed=seed)
    cfg = wl.coupled_config(pkg, nx, ny, nz, dissolution=True)
    bio = wl.seed_biomass(mask, seed + 1)
    mineral = wl.seed_mineral(mask, seed + 2, cfg.max_precip_rho)
    return cfg, mask, bio, mineral


def fluid_counts(cfg, mask):
    fluid = np.isin(mask, list(cfg.pore_codes)[:cfg.n_pore_codes] + list(cfg.bio_codes)[:cfg.n_bio_codes])
    return int(fluid[1:-1].sum()), int(fluid.sum())


def coupled_step(lat, i, geometry=False):
    """One coupled step: transport, the amortised flow re-solve (500 steps per
    200 transport steps), and, when `geometry`, the node conversions
    (precipitation seals, dissolution reopens) with the dynamics switch and
    the velocity re-coupling.  Returns the voxels converted."""
    lat.step(1)
    lat.flow_steps(2 if i % 2 == 0 else 3)
    if not geometry:
        return 0
    changed = lat.precip_convert() + lat.dissol_convert()
    lat.update_dynamics()
    lat.couple_velocity()
    return changed


# ----------------------------------------------------------------- CPU legs
def cpu_coupled(steps, seed=5):
    """The FP64 oracle (OpenMP, all host cores) on a bounded sample of the
    coupled workload: returns (MLUPS, seconds, threads, sample text)."""
    pkg, wl = load_pkg(), load_workloads()
    from oracle import oracle as o
    cfg, mask, bio, mineral = coupled_setup(pkg, wl, CPU_SAMPLE, seed)
    fl = o.Flow(cfg, mask)
    fl.step(50)
    _, u = fl.macro()
    tr = o.Transport(cfg, mask, u=u)
    tr.set_biomass(0, bio)
    tr.set_conc(8, mineral)
    tr.step(1)
    t0 = time.perf_counter()
    for i in range(steps):
        tr.step(1)
        fl.step(2 if i % 2 == 0 else 3)
    dt = time.perf_counter() - t0
    N = int(np.prod(CPU_SAMPLE))
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = "%dx%dx%d sites (same chemistry, porosity, step schedule), %d coupled steps" % (
        CPU_SAMPLE[0], CPU_SAMPLE[1], CPU_SAMPLE[2], steps)
    return N * steps / dt / 1e6, dt, threads, sample


def cpu_pcf(n=16384):
    """The oracle's PCF + Anderson (the reference's code restated; identical
    iterates, tests/test_oracle_pcf.py) on the first n voxels of the
    speciation batch, all host threads: solves per second."""
    pkg, wl = load_pkg(), load_workloads()
    from oracle import oracle as o
    S, logk, cs = wl.tableau(5, 9, seed=4)
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, cs, max_iter=200, tol=1e-10, warm_iter=6)
    T, _, _, _ = wl.speciation_batch(S, logk, n, seed=302)
    c = wl.cold_species(S, T, cs)
    t0 = time.perf_counter()
    _, it, cv = o.pcf_batch(sys_, c)
    dt = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"solves_per_s": n / dt, "cores": threads, "kind": "port", "mean_iters": float(it.mean()),
            "converged": float(cv.mean()), "sample": "%d voxels of the same batch" % n}


def run_reference(args, rank):
    if rank != 0:
        return
    steps = max(args.steps, 1)
    mlups, dt, threads, sample = cpu_coupled(steps)
    line = {"impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS", "n_gpus": args.gpus,
            "steps": steps, "warmup": args.warmup, "ms_per_step": dt / steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_block(),
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": threads, "kind": "port",
                             "sample": sample + "; the reference's own LBM path needs Palabos v2.3.0, which is "
                                                "not vendored, so its CPU restatement runs instead"},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_block():
    return {"workload": "coupled sphere pack %dx%dx%d (nx incl. 2 boundary planes), porosity 0.35, radii 5-10; "
                        "D3Q19 flow (2.5 steps amortised) + D3Q7 ADR of 8 mobile solutes + 1 mineral, dual-Monod "
                        "kinetics, surface precipitation, 3-component Newton speciation per pore voxel"
                        % FULL,
            "nx": FULL[0], "ny": FULL[1], "nz": FULL[2], "sites": int(np.prod(FULL)),
            "l2": "inputs larger than L2 (about 13 GB of state), no flush",
            "parallelism": "one domain per GPU (weak scaling, no data-path collective)"}


# ----------------------------------------------------------------- speciation
def speciation_bench(pkg, wl, stream, n_train=1 << 20, n_test=1 << 21):
    import torch
    S, logk, cs = wl.tableau(5, 9, seed=4)
    sys_ = pkg.EqSystem()
    pkg.set_eq_system(sys_, S, logk, cs, max_iter=200, tol=1e-10, warm_iter=6)
    eq = pkg.EqSolver(sys_, stream=stream)
    dev = torch.device("cuda")
    Ttr, _, _, _ = wl.speciation_batch(S, logk, n_train, seed=301)
    Tte, _, _, acc = wl.speciation_batch(S, logk, n_test, seed=302)
    f64 = dict(dtype=torch.float64, device=dev)
    dT = torch.tensor(Ttr, **f64)
    dC = torch.tensor(wl.cold_species(S, Ttr, cs), **f64)
    dX = torch.zeros((n_train, 5), **f64)
    dI = torch.zeros(n_train, dtype=torch.int32, device=dev)
    dS = torch.zeros(n_train, dtype=torch.uint8, device=dev)
    t0 = time.perf_counter()
    eq.solve_device(dT.data_ptr(), dC.data_ptr(), dX.data_ptr(), dI.data_ptr(), dS.data_ptr(), n_train,
                    pkg.EQ_START_COLD)
    ok = (dS == 0)
    Tk, Xk = dT[ok].contiguous(), dX[ok].contiguous()
    loss = eq.train_device(Tk.data_ptr(), Xk.data_ptr(), int(Tk.shape[0]), epochs=30, batch=4096, lr=3e-3, seed=7)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    eT = torch.tensor(Tte, **f64)
    eC = torch.tensor(wl.cold_species(S, Tte, cs), **f64)
    res = {}
    for name, start in (("cold", pkg.EQ_START_COLD), ("learned", pkg.EQ_START_LEARNED)):
        X = torch.zeros((n_test, 5), **f64)
        I = torch.zeros(n_test, dtype=torch.int32, device=dev)
        St = torch.zeros(n_test, dtype=torch.uint8, device=dev)
        eq.solve_device(eT.data_ptr(), eC.data_ptr(), X.data_ptr(), I.data_ptr(), St.data_ptr(), n_test, start)
        times = []
        for _ in range(3):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s0.record()
            eq.solve_device(eT.data_ptr(), eC.data_ptr(), X.data_ptr(), I.data_ptr(), St.data_ptr(), n_test, start)
            s1.record()
            torch.cuda.synchronize()
            times.append(s0.elapsed_time(s1))
        ms = min(times)
        st = St.cpu().numpy()
        res[name] = {"ms": ms, "solves_per_s": n_test / (ms * 1e-3), "mean_iters": float(I.float().mean().item()),
                     "converged": float((st <= 1).mean()), "fell_back": float((st == 1).mean()),
                     "x": X, "ok": St <= 1}
    # where the learned time goes: the network alone, and Newton from its
    # start and from the converged roots (the cost floor of one check)
    def timed(fn, reps=3):
        ts = []
        for _ in range(reps):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            s0.record()
            fn()
            s1.record()
            torch.cuda.synchronize()
            ts.append(s0.elapsed_time(s1))
        return min(ts)
    Xp = torch.zeros((n_test, 5), **f64)
    X = torch.zeros((n_test, 5), **f64)
    I = torch.zeros(n_test, dtype=torch.int32, device=dev)
    St = torch.zeros(n_test, dtype=torch.uint8, device=dev)
    res["breakdown_ms"] = {"network": timed(lambda: eq.predict_device(eT.data_ptr(), Xp.data_ptr(), n_test))}
    for name, start_x in (("newton_from_network", Xp), ("newton_from_root", res["cold"]["x"])):
        def run(start_x=start_x):
            X.copy_(start_x)
            eq.solve_device(eT.data_ptr(), eC.data_ptr(), X.data_ptr(), I.data_ptr(), St.data_ptr(), n_test,
                            pkg.EQ_START_GIVEN)
        res["breakdown_ms"][name] = timed(run)
        res["breakdown_ms"][name + "_mean_iters"] = float(I.float().mean().item())
    # the reference's live solver (PCF + Anderson) on the same voxels, from
    # their cold species vectors (calculate_species_concentrations)
    Pout = torch.zeros_like(eC)
    PI = torch.zeros(n_test, dtype=torch.int32, device=dev)
    PC = torch.zeros(n_test, dtype=torch.uint8, device=dev)
    pcf_run = lambda: eq.pcf_device(eC.data_ptr(), Pout.data_ptr(), PI.data_ptr(), PC.data_ptr(), n_test)
    pcf_run()
    pms = timed(pcf_run)
    res["pcf"] = {"ms": pms, "solves_per_s": n_test / (pms * 1e-3), "mean_iters": float(PI.float().mean().item()),
                  "converged": float(PC.float().mean().item()),
                  "solver": "PCF + Anderson depth 4, ||f||_2 < 1e-10, <= 200 iterations (the reference's settings)"}
    # same roots and residuals where both converged
    from_cold, from_learned = res["cold"].pop("x"), res["learned"].pop("x")
    both = res["cold"].pop("ok") & res["learned"].pop("ok")
    diff = (from_cold - from_learned).abs().max(dim=1).values[both]
    res["max_abs_logdiff_both_converged"] = float(diff.max().item()) if diff.numel() else None
    res["speedup_learned_vs_cold"] = res["cold"]["ms"] / res["learned"]["ms"]
    res.update({"n_solves": n_test, "n_train_pairs": int(Tk.shape[0]), "train_s": train_s, "final_loss": loss,
                "tableau": "5 components x 14 species, logK U[-14,14], stoichiometry in [-2,2] (negative only on "
                           "the pH-like component), totals 1e-6..1e-1, free H 1e-9..1e-5; acceptance %.3f" % acc,
                "residual": "max_j |S^T c - T|_j / (|S|^T c)_j <= 1e-10"})
    eq.close()
    return res


# ----------------------------------------------------------------- other workloads
def transport_roofline(ms, launches, n_fluid_int, bytes_per_site, n_interior, peak, peak_kind, kernel):
    if not launches:
        return None
    b = n_fluid_int * bytes_per_site + n_interior
    a = b / (ms / launches * 1e-3) / 1e9
    return {"kernel": kernel, "bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s", "frac": a / peak,
            "peak_source": peak_kind + " (hbm_gbs)", "algorithmic_bytes_per_launch": b,
            "avg_launch_ms": ms / launches, "traffic": None}


def surrogate_bench(pkg, wl, stream, steps=20, warmup=3, shape=(256, 256, 256)):
    """The surrogate-rate workload: 256^3 sphere pack (porosity 0.4), two
    organisms each with a 3 -> 20 tanh -> 20 tanh -> 4 network (mapminmax,
    weights ~N(0, 0.3)), six solutes, the networks evaluated per voxel in the
    step; transport step MLUPS and its roofline, and the FP64 oracle on a 64^3
    sample of the same workload."""
    import torch
    nx, ny, nz = shape
    mask = wl.sphere_pack(nx, ny, nz, 0.40, 4.0, 8.0, seed=31)
    cfg = wl.surrogate_config(pkg, nx, ny, nz)
    nets = wl.surrogate_nets(pkg)
    b = [wl.seed_biomass(mask, 32 + m, frac=0.3, lo=0.005, hi=0.05) for m in range(2)]
    lat = pkg.Lattice(cfg, stream=stream)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(200)
    lat.couple_velocity()
    for slot in range(2):
        lat.set_surrogate(slot, nets[slot])
    lat.ade_init()
    for m in range(2):
        lat.set_field(pkg.FIELD_BIOMASS, m, b[m])
    for _ in range(warmup):
        lat.step(1)
    torch.cuda.synchronize()
    lat.timing(True)
    lat.timing_read(pkg.KERNEL_ADE_MAIN)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        lat.step(1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ade_ms, ade_n = lat.timing_read(pkg.KERNEL_ADE_MAIN)
    compiled = lat.get_option(pkg.OPT_COMPILED_CHEM) == pkg.CHEM_SURROGATE2
    lat.timing(False)
    lat.close()
    N = mask.size
    n_fluid_int, _ = fluid_counts(cfg, mask)
    peak, peak_kind = peaks()
    how = ("one launch: ade_fast_kernel with the networks' weights in its parameter space" if compiled
           else "reaction + streaming launches")
    roof = transport_roofline(ade_ms, ade_n, n_fluid_int, 6 * 56 + 12 + 2 * 8, N - 2 * ny * nz, peak, peak_kind,
                              "transport step with the per-voxel networks (%s)" % how)
    return {"workload": "surrogate: %dx%dx%d sphere pack, porosity 0.4, 2 organisms x (3->20->20->4), 6 solutes"
                        % shape, "mlups": N * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps,
            "roofline": roof}


def c1_bench(pkg, wl, stream, flow_steps=2000, ade_steps=1000, cpu=True):
    """The 64^3 flow + transport configuration as stated: spheres r 4-8 to
    porosity 0.40 in 64^3 voxels (plus the two boundary planes), rho
    1.001 / 1.000, tau 0.8, 2000 flow steps; then one solute, tau 0.7,
    Dirichlet C = 1 inlet, zero-gradient outlet, 1000 transport steps.  Flow
    and transport MLUPS (all sites) on the GPU, and the FP64 oracle on the
    same domain for 100 + 100 steps."""
    import torch
    nx, ny, nz = 66, 64, 64
    mask = wl.sphere_pack(nx, ny, nz, 0.40, 4.0, 8.0, seed=101)
    cfg = pkg.make_config(nx, ny, nz, tau_ns=0.8, rho_in=1.001, rho_out=1.0,
                          solutes=[{"tau": 0.7, "c0": 0.0, "left": "D", "left_value": 1.0, "right": "N"}])
    lat = pkg.Lattice(cfg, stream=stream)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(20)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    torch.cuda.synchronize()
    e[0].record()
    lat.flow_steps(flow_steps)
    e[1].record()
    lat.couple_velocity()
    lat.ade_init()
    lat.step(5)
    torch.cuda.synchronize()
    e[2].record()
    lat.step(ade_steps)
    e[3].record()
    torch.cuda.synchronize()
    fms, ams = e[0].elapsed_time(e[1]), e[2].elapsed_time(e[3])
    outlet = float(lat.field(pkg.FIELD_CONC, 0).reshape(nx, ny, nz)[nx - 2].mean())
    lat.close()
    N = mask.size
    res = {"workload": "64^3 spheres r 4-8, porosity 0.40, tau 0.8, 2000 flow steps; one solute, tau 0.7, "
                       "1000 transport steps (FP32 populations)",
           "flow_mlups": N * flow_steps / (fms * 1e-3) / 1e6, "transport_mlups": N * ade_steps / (ams * 1e-3) / 1e6,
           "flow_ms": fms, "transport_ms": ams, "outlet_mean_after": outlet}
    if not cpu:
        return res
    from oracle import oracle as o
    fl = o.Flow(cfg, mask)
    t0 = time.perf_counter()
    fl.step(100)
    cf = time.perf_counter() - t0
    _, u = fl.macro()
    tr = o.Transport(cfg, mask, u=u)
    t0 = time.perf_counter()
    tr.step(100)
    ca = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    res["cpu_baseline"] = {"flow_mlups": N * 100 / cf / 1e6, "transport_mlups": N * 100 / ca / 1e6,
                           "unit": "MLUPS", "cores": threads, "kind": "port",
                           "sample": "the same 66x64x64 domain, 100 flow + 100 transport steps (FP64 oracle)"}
    return res


def cpu_surrogate(steps=40, shape=(64, 64, 64)):
    pkg, wl = load_pkg(), load_workloads()
    from oracle import oracle as o
    nx, ny, nz = shape
    mask = wl.sphere_pack(nx, ny, nz, 0.40, 4.0, 8.0, seed=31)
    cfg = wl.surrogate_config(pkg, nx, ny, nz)
    nets = wl.surrogate_nets(pkg)
    fl = o.Flow(cfg, mask)
    fl.step(30)
    _, u = fl.macro()
    tr = o.Transport(cfg, mask, u=u)
    tr.set_surrogates(nets)
    for m in range(2):
        tr.set_biomass(m, wl.seed_biomass(mask, 32 + m, frac=0.3, lo=0.005, hi=0.05))
    t0 = time.perf_counter()
    tr.step(steps)
    dt = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": mask.size * steps / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": "%dx%dx%d of the same workload, %d transport steps" % (nx, ny, nz, steps)}


def cpu_biotic_ca(steps=40, shape=(64, 64, 64)):
    """The FP64 oracle on a 64^3 sample of the biotic + CA workload: transport
    step and CA block per step."""
    pkg, wl = load_pkg(), load_workloads()
    from oracle import oracle as o
    nx, ny, nz = shape
    mask = wl.walled_pack(nx, ny, nz, 0.35, 5.0, 10.0, seed=21)
    cfg = wl.biotic_config(pkg, nx, ny, nz)
    fl = o.Flow(cfg, mask)
    fl.step(30)
    _, u = fl.macro()
    tr = o.Transport(cfg, mask, u=u)
    tr.set_biomass(0, wl.seed_biomass(mask, 22))
    tr.ca_init()
    tr.ca_update_mask()
    t0 = time.perf_counter()
    for _ in range(steps):
        tr.step(1)
        tr.ca_redistribute()
    dt = time.perf_counter() - t0
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": mask.size * steps / dt / 1e6, "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": "%dx%dx%d of the same workload, %d steps (transport + CA block)" % (nx, ny, nz, steps)}


def learned_step_bench(pkg, wl, stream, shape=(256, 128, 128), steps=40, interval=10):
    """The learned warm start inside the coupled step: the network is trained
    on the device every `interval` steps on the step's own Newton pairs; then
    every voxel forgets its previous solution and one more step runs, started
    from the network, against the same step started cold.  Newton
    iterations per reactive voxel of that step, the Newton time (the
    transport step), and the training time."""
    import torch
    cfg, mask, bio, mineral = coupled_setup(pkg, wl, shape, seed=15)
    react = (mask == 2)
    react[0] = react[-1] = False
    res = {}
    for learn in (True, False):
        lat = pkg.Lattice(cfg, stream=stream)
        lat.upload_mask(mask)
        lat.flow_init()
        lat.flow_steps(100)
        lat.couple_velocity()
        lat.ade_init()
        lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
        lat.set_field(pkg.FIELD_CONC, 8, mineral)
        if learn:
            lat.set_option(pkg.OPT_EQ_LEARN, interval)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(steps):
            lat.step(1)
        torch.cuda.synchronize()
        run_s = time.perf_counter() - t0
        lat.set_option(pkg.OPT_EQ_FORGET, 1)
        lat.timing(True)
        lat.timing_read(pkg.KERNEL_ADE_MAIN)
        lat.step(1)
        ms, n = lat.timing_read(pkg.KERNEL_ADE_MAIN)
        lat.timing(False)
        it = lat.field(pkg.FIELD_EQ_ITERS).reshape(mask.shape)[react]
        res["learned" if learn else "cold"] = {"mean_iters": float(it.mean()), "max_iters": int(it.max()),
                                               "step_ms": ms / max(n, 1), "run_s": run_s}
        if learn:
            res["trainings"] = lat.get_option(pkg.OPT_EQ_LEARN_TRAININGS)
        lat.close()
    res["workload"] = ("coupled %dx%dx%d, network trained every %d steps over %d steps on 1/16 of the converged "
                       "voxels' pairs, then one step with every voxel's history cleared" % (shape + (interval, steps)))
    res["training_overhead_s"] = res["learned"]["run_s"] - res["cold"]["run_s"]
    return res


# ----------------------------------------------------------------- main arm
def biotic_ca_bench(pkg, wl, stream, steps=20, warmup=3, shape=(128, 128, 128)):
    """The biotic workload with the cellular-automaton biofilm: 128^3 sphere
    pack (porosity 0.35, radii 5-10) in a duct with bounce-back walls on the
    y / z faces and sealed pores filled, four solutes, dual-Monod kinetics,
    biomass 10-50 on 2% of the wall-adjacent pore voxels, Bmax 100.  Each step
    is the transport step and the CA block (its mask / total update and
    maximum on every step; push sweeps when a voxel exceeds Bmax).  The CA
    block is also timed on its own on the same state with the biomass scaled
    x5, so that about half the colonies exceed Bmax and spread."""
    import torch
    nx, ny, nz = shape
    mask = wl.walled_pack(nx, ny, nz, 0.35, 5.0, 10.0, seed=21)
    cfg = wl.biotic_config(pkg, nx, ny, nz)
    bio = wl.seed_biomass(mask, 22)
    lat = pkg.Lattice(cfg, stream=stream)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(200)
    lat.couple_velocity()
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
    lat.ca_update_mask()
    for _ in range(warmup):
        lat.step(1)
        lat.ca_redistribute()
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * steps + 2)]
    ev[0].record()
    for i in range(steps):
        lat.step(1)
        ev[1 + 2 * i].record()
        lat.ca_redistribute()
        ev[2 + 2 * i].record()
    ev[-1].record()
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[-1])
    ca_ms = sum(ev[1 + 2 * i].elapsed_time(ev[2 + 2 * i]) for i in range(steps))
    N = mask.size
    # one CA block with work: the seeded colonies at x5
    b = lat.field(pkg.FIELD_BIOMASS, 0) * 5.0
    lat.set_field(pkg.FIELD_BIOMASS, 0, b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    st, sweeps, changes, bmax = lat.ca_redistribute()
    e1.record()
    torch.cuda.synchronize()
    block_ms = e0.elapsed_time(e1)
    over = int((b > cfg.ca_bmax).sum())
    lat.close()
    n_fluid_int, _ = fluid_counts(cfg, mask)
    peak, peak_kind = peaks()
    # the transport step of this workload alone (steps without the CA block)
    roof = transport_roofline(ms - ca_ms, steps, n_fluid_int, 4 * 56 + 12 + 8, N - 2 * ny * nz, peak, peak_kind,
                              "transport step (4 solutes, dual Monod) of the biotic + CA workload")
    return {"workload": "biotic + CA: %dx%dx%d sphere pack, porosity 0.35, radii 5-10, walled duct, sealed pores "
                        "filled; 4 solutes, dual Monod, "
                        "biomass 10-50 on 2%% of wall-adjacent pore voxels, Bmax 100, fraction push" % shape,
            "mlups": N * steps / (ms * 1e-3) / 1e6, "ms_per_step": ms / steps, "ca_ms_per_step": ca_ms / steps,
            "roofline": roof,
            "ca_block": {"status": st, "voxels_over_bmax": over, "sweeps": sweeps, "mask_changes": changes,
                         "ms": block_ms, "ms_per_sweep": block_ms / max(sweeps, 1), "max_after": bmax}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-speciation", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-biotic", action="store_true")
    ap.add_argument("--shape", default=None, help="override nx,ny,nz (development only)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    args.warmup = max(args.warmup, 3)
    global FULL
    if args.shape:
        FULL = tuple(int(v) for v in args.shape.split(","))
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    # a dedicated stream: the library's kernels and the torch events that time
    # them share it (the legacy default stream has handle 0, which the C ABI
    # reads as "create your own")
    torch.cuda.set_stream(torch.cuda.Stream())
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    pkg, wl = load_pkg(), load_workloads()
    stream = torch.cuda.current_stream().cuda_stream
    cfg, mask, bio, mineral = coupled_setup(pkg, wl, FULL, seed=5 + rank)
    n_fluid_int, n_fluid = fluid_counts(cfg, mask)
    N = int(np.prod(FULL))
    lat = pkg.Lattice(cfg, stream=stream)
    lat.upload_mask(mask)
    lat.flow_init()
    lat.flow_steps(200)
    lat.couple_velocity()
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, bio)
    lat.set_field(pkg.FIELD_CONC, 8, mineral)
    for i in range(args.warmup):
        coupled_step(lat, i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    lat.timing(True)
    lat.timing_read(pkg.KERNEL_ADE_MAIN)
    lat.timing_read(pkg.KERNEL_FLOW_STEP)
    l0 = lat.launch_count()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.nvtx.range_push("timed")       # lets a profiler select the timed launches
    e0.record()
    converted = 0
    for i in range(args.steps):
        # the geometry block of every 200 steps falls on the first timed step
        # (with fewer than 200 timed steps it is counted more often than the
        # workload runs it, never less)
        converted += coupled_step(lat, args.warmup + i, geometry=(i % 200 == 0))
    e1.record()
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launches = lat.launch_count() - l0
    ade_ms, ade_n = lat.timing_read(pkg.KERNEL_ADE_MAIN)
    flow_ms, flow_n = lat.timing_read(pkg.KERNEL_FLOW_STEP)
    lat.timing(False)
    clk = clocks.stop()
    ms = max_over_ranks(ms, dist, "cuda")
    if world > 1:
        dist.barrier()
    ms_per_step = ms / args.steps
    value = job_mlups(N, world, args.steps, ms)
    out = {"metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32 populations, f64 speciation", "data": "synthetic (seeded sphere pack)",
           "config": config_block(), "fluid_mlups": n_fluid * world * args.steps / (ms * 1e-3) / 1e6,
           "gpu_launches": int(launches), "clocks": clk,
           "geometry": {"blocks_timed": (args.steps + 199) // 200, "voxels_converted": int(converted),
                        "block": "precipitation seal + dissolution reopen + dynamics switch + velocity re-coupling"},
           "transport_launch": "one launch per step (compiled chemistry: %s)" % (
               "coupled carbonate" if lat.get_option(pkg.OPT_COMPILED_CHEM) == pkg.CHEM_COUPLED else "none")}
    # roofline of the dominant work: the transport step, whose reaction and
    # streaming launches run slab-interleaved on two streams and are timed
    # together (one event pair per step on the context's stream)
    peak, peak_kind = peaks()
    ade_bytes = n_fluid_int * ADE_BYTES_PER_FLUID_SITE + (N - 2 * FULL[1] * FULL[2])
    if ade_n:
        achieved = ade_bytes / (ade_ms / ade_n * 1e-3) / 1e9
        tps = traffic_from_profile("ade_fast")
        out["roofline"] = {"kernel": "transport step: ade_fast_kernel (gather, FP64 reaction chain, collide, "
                                     "stream in one launch)", "bound": "hbm",
                           "limiter": "issue latency of the FP64 Newton chain at 24% warp occupancy (ncu); the "
                                      "same launch without the chain streams at ~0.6 of the HBM peak",
                           "target_frac": 0.60,
                           "achieved": achieved, "peak": peak,
                           "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind + " (hbm_gbs)",
                           "algorithmic_bytes_per_launch": ade_bytes, "avg_launch_ms": ade_ms / ade_n,
                           "traffic": (tps * n_fluid_int) if tps else None,
                           "share_of_step": ade_ms / ms if ms else None}
    if flow_n:
        n_bgk = n_fluid
        fb = n_bgk * FLOW_BYTES_PER_BGK_SITE + N
        out["flow_kernel"] = {"achieved_gbs": fb / (flow_ms / flow_n * 1e-3) / 1e9, "avg_launch_ms": flow_ms / flow_n,
                              "launches": flow_n, "share_of_step": flow_ms / ms if ms else None}
    # end to end through the C ABI with pinned host buffers
    if not args.no_e2e:
        out["e2e"] = e2e_run(pkg, torch, cfg, mask, bio, mineral, args.steps, stream, world)
    lat.close()
    if rank == 0 and world == 1 and not args.no_speciation:
        out["speciation"] = speciation_bench(pkg, wl, stream)
    if rank == 0 and world == 1 and not args.no_biotic:
        out["biotic_ca"] = biotic_ca_bench(pkg, wl, stream)
        out["surrogate"] = surrogate_bench(pkg, wl, stream)
        out["flow_transport_64"] = c1_bench(pkg, wl, stream, cpu=not args.no_cpu)
        out["learned_step"] = learned_step_bench(pkg, wl, stream)
    if rank == 0 and world == 1 and not args.no_cpu:
        cm, cdt, threads, sample = cpu_coupled(40)
        out["cpu_baseline"] = {"value": cm, "unit": "MLUPS", "cores": threads, "kind": "port", "sample": sample}
        if "speciation" in out:
            out["speciation"]["pcf"]["cpu"] = cpu_pcf()
        if "biotic_ca" in out:
            out["biotic_ca"]["cpu_baseline"] = cpu_biotic_ca()
            out["surrogate"]["cpu_baseline"] = cpu_surrogate()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(out), flush=True)


def e2e_run(pkg, torch, cfg, mask, bio, mineral, steps, stream, world):
    """The same job through the public C ABI with pinned host buffers: upload
    the geometry and the biomass, initialise, run the steps, read every solute
    field back; the copies are inside the timed region."""
    N = mask.size
    h_mask = torch.from_numpy(np.ascontiguousarray(mask.reshape(-1))).pin_memory().numpy()
    h_bio = torch.from_numpy(np.ascontiguousarray(bio.reshape(-1))).pin_memory().numpy()
    h_min = torch.from_numpy(np.ascontiguousarray(mineral.reshape(-1))).pin_memory().numpy()
    h_out = torch.empty((cfg.n_solutes, N), dtype=torch.float64).pin_memory().numpy()
    lat = pkg.Lattice(cfg, stream=stream)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lat.upload_mask(h_mask)
    lat.flow_init()
    lat.couple_velocity()
    lat.ade_init()
    lat.set_field(pkg.FIELD_BIOMASS, 0, h_bio)
    lat.set_field(pkg.FIELD_CONC, 8, h_min)
    for i in range(steps):
        coupled_step(lat, i, geometry=(i % 200 == 0))
    for s in range(cfg.n_solutes):
        lat._c(lat.lib.cl_get_field(lat.h, pkg.FIELD_CONC, s, pkg._ptr(h_out[s])), "cl_get_field")
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    lat.close()
    import torch.distributed as dist
    dt = max_over_ranks(dt, dist, "cuda")
    h2d = h_mask.nbytes + h_bio.nbytes + h_min.nbytes
    d2h = h_out.nbytes
    return {"value": job_mlups(N, world, steps, dt * 1e3), "unit": "MLUPS", "h2d_bytes_per_step": h2d // steps,
            "d2h_bytes_per_step": d2h // steps,
            "includes": "geometry and biomass upload, initialisation, the steps (flow develops inside the "
                        "amortised re-solve), and the read-back of every solute field, amortised over the steps"}


if __name__ == "__main__":
    main()
