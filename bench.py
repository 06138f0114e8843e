"""Benchmark of the coupled gauge + NRQCD timestep on B200.

One step = one NRQCDField%Update (Crank-Nicolson step of quark and
antiquark, 12 propagator columns) followed by one GaugeConfiguration%Update
(leapfrog), the driver order of src/main.f90:344-348.

Workload (plain FP64 at 64^3): transverse-polarised occupation initial
condition n0 = 1, aQ = 0.5, coupling 0, ranlxd seed 1, links = 1; a0 = 0.05,
a_s = 1; point sources at the origin; aM = 1.0, Wilson coefficients 1;
Krylov residual 1e-12.  Synthetic, seeded fields; the working set (~3 GB)
exceeds the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--size L]

For N > 1 (launched with torch.distributed.run) every rank evolves its own
independent lattice (an ensemble member, seed 1 + rank); there is no
data-path collective.  Rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# the CPU legs' OpenMP worker threads sleep between parallel regions instead
# of spinning, so they do not take host cores from the GPU-timed loops that
# read results back every iteration
os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")

METRIC = "site-updates/s per 64^3 gauge+NRQCD step; CN s/step vs FP64 plain at ≤1e-10"
MASS = 1.0
WILSON = [1.0, 1.0, 1.0, 1.0]
A = (0.05, 1.0, 1.0, 1.0)
TOL = 1e-12
# DRAM bytes per site of an average stencil launch of a plain 64^3 update
# (dram__bytes_read.sum + dram__bytes_write.sum, one ncu capture of the
# update's 9 launches), by NRQ_STENCIL_* index: the tensor-core stencil (2
# residual, 4 v and 3 t launches: 10,773, 7,760 and 6,377 B/site) and the
# FMA stencil (1 right-hand side, 2 residual, 3 v and 3 t launches: 7,573,
# 10,413, 7,500 and 6,199 B/site)
STENCIL_DRAM_BYTES_PER_SITE = {2: 7968.0, 3: 7722.0}
# FP64 arithmetic of the leapfrog force per site: 3 directions x (4 staples
# of 2 products + the product with the link) = 27 complex 3x3 products of
# 27 complex multiply-adds, 4 real FMAs each, 2 flops per FMA
LEAPFROG_FORCE_FLOPS_PER_SITE = 27 * 27 * 4 * 2
# FP64 stencils of the solver, by NRQ_STENCIL_* index
STENCIL_NAMES = {0: "k_cn_mv2 (register-tiled)", 1: "k_cn_mv3 (TMA-staged)", 2: "k_cn_mv4 (FP64 tensor cores)",
                 3: "k_cn_mv5 (FP64 FMA on cached blocks)"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=30)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--size", type=int, default=64)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-forms", action="store_true")
    p.add_argument("--no-ensemble", action="store_true")
    p.add_argument("--only-ensemble", action="store_true", help="print only the batching-ensemble JSON")
    p.add_argument("--ensemble-members", default=None,
                   help="with --only-ensemble: members as EXTENTxCOUNT[,...] (default the C4 ensemble)")
    p.add_argument("--ensemble-sources", type=int, default=None,
                   help="with --only-ensemble: point sources per member and mass (default 16)")
    p.add_argument("--ensemble-no-learned", action="store_true",
                   help="with --only-ensemble: skip the learned-guess leg")
    p.add_argument("--only-forms", action="store_true", help="print only the CN-forms JSON")
    p.add_argument("--forms-sizes", type=int, nargs="+", default=list(FORMS_SIZES))
    p.add_argument("--no-drift", action="store_true")
    p.add_argument("--no-thermal", action="store_true")
    p.add_argument("--no-gluon", action="store_true")
    p.add_argument("--only-gluon", action="store_true", help="print only the gluon-distribution JSON")
    p.add_argument("--only-thermal", action="store_true", help="print only the thermal initial-condition JSON")
    p.add_argument("--stencil", default="timed", choices=["timed", "register", "tma", "tensor", "fma"],
                   help="FP64 stencil of the headline step (default: the solver's timed choice)")
    p.add_argument("--only-drift", action="store_true", help="print only the precision-drift JSON")
    p.add_argument("--two-pass", action="store_true",
                   help="headline step: the two-pass BiCGStab update in place of the merged one")
    p.add_argument("--history-depth", type=int, default=None,
                   help="headline step: history vectors of the plain solve's start (1-4; default the library's)")
    return p.parse_args()


def workload_config(L, n_gpus):
    return {"workload": f"coupled CN(12 columns)+leapfrog step, plain FP64, {L}^3 periodic lattice",
            "lattice": [L, L, L], "spacings": list(A), "mass": MASS, "wilson_coefficients": WILSON,
            "krylov_tol": TOL, "initial_condition": "transverse box n0=1 aQ=0.5 g=0 seed=1(+rank), U=1",
            "sources": "point source at lattice index 1 (quark and antiquark)",
            "l2": "inputs larger than L2 (working set ~3 GB > 126 MB)",
            "parallelism": f"replicas x{n_gpus} (independent ensemble members)"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clocks and clock-event reasons of this rank's GPU during the timed
    region: NVML polled every 10 ms from a thread (started before the
    warm-up, so that the timed region is covered from its first
    millisecond; mark() and stop() bound the window), else nvidia-smi at
    50 ms.  Reads only; changes no setting of the GPU."""
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.samples = []  # (time, sm MHz, max MHz, reasons)
        self.t0 = None
        self.proc = None
        self.stop_ev = threading.Event()
        self.thread = None
        self.source = None

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        p = torch.cuda.get_device_properties(self.dev)
        bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        try:
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.dev)

    def start(self):
        try:
            nv, h = self._nvml_handle()
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
            smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))

            def poll():
                while not self.stop_ev.is_set():
                    try:
                        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                        r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                        self.samples.append((time.perf_counter(), sm, smax,
                                             {k for k, bit in bits.items() if r & bit}))
                    except Exception:
                        pass
                    self.stop_ev.wait(0.01)
            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
            self.source = "nvml"
            return
        except Exception:
            pass
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "50", "-i", str(self.dev)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)

            def read():
                for line in self.proc.stdout:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) < 9:
                        continue
                    try:
                        sm, smax = float(parts[1]), float(parts[2])
                    except ValueError:
                        continue
                    self.samples.append((time.perf_counter(), sm, smax,
                                         {nm for nm, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}))
            self.thread = threading.Thread(target=read, daemon=True)
            self.thread.start()
            self.source = "nvidia-smi"
        except Exception:
            self.proc = None

    def mark(self):
        """The timed region begins now."""
        self.t0 = time.perf_counter()

    def stop(self):
        t1 = time.perf_counter()
        if self.source is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        time.sleep(0.03)  # the sample that straddles the end
        self.stop_ev.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        t0 = self.t0 if self.t0 is not None else 0.0
        inside = [s for s in self.samples if t0 <= s[0] <= t1 + 0.02]
        sm = [s[1] for s in inside]
        reasons = set().union(*[s[3] for s in inside]) if inside else set()
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(s[2] for s in inside) if inside else None,
                "sm_min_mhz": min(sm) if sm else None, "reasons": sorted(reasons), "samples": len(sm),
                "source": self.source}


# ------------------------------------------------------------------ reference arm
def run_reference(args, rank):
    """The reference's CPU algorithm (oracle restatement) on the host cores."""
    if rank != 0:
        return
    from oracle import oracle as oc
    # rank 0 runs alone on the host: every core it may use (a launcher sets
    # OMP_NUM_THREADS=1 per rank)
    oc.set_num_threads(len(os.sched_getaffinity(0)))
    L = args.size
    n = (L, L, L)
    V = L ** 3
    links, ef = oc.transverse_box(n, A, 0.5, 1.0, 0.0, 1, identity_links=True)
    q = oc.single_point(n, 1)
    an = oc.single_point(n, 1)

    def step():
        oc.cn_update(n, A, links, ef, MASS, WILSON, 1.0, q, an, tol=TOL)
        oc.gauge_update(n, A, links, ef, 1.0)

    t0 = time.perf_counter()
    step()  # one warm-up step (the CPU path has no compilation or cache state to warm)
    t_first = time.perf_counter() - t0
    budget = 150.0
    steps = max(1, min(args.steps, int(budget / max(t_first, 1e-3))))
    t0 = time.perf_counter()
    for _ in range(steps):
        step()
    dt = time.perf_counter() - t0
    value = V * steps / dt
    cores = oc.num_threads()
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "site-updates/s",
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * dt / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(L, 1),
            "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": cores, "kind": "port",
                             "sample": f"{steps} coupled {L}^3 steps after 1 warm-up step (budget {budget:.0f} s); "
                                       "FP64 C restatement of the reference algorithm (OpenMP), GMRES(30) to 1e-12"},
            "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(L):
    """Bounded CPU-baseline sample (one coupled step of the same workload)."""
    from oracle import oracle as oc
    n = (L, L, L)
    links, ef = oc.transverse_box(n, A, 0.5, 1.0, 0.0, 1, identity_links=True)
    q = oc.single_point(n, 1)
    an = oc.single_point(n, 1)
    t0 = time.perf_counter()
    oc.cn_update(n, A, links, ef, MASS, WILSON, 1.0, q, an, tol=TOL)
    oc.gauge_update(n, A, links, ef, 1.0)
    dt = time.perf_counter() - t0
    return {"value": L ** 3 / dt, "unit": "site-updates/s", "cores": oc.num_threads(), "kind": "port",
            "sample": f"1 coupled {L}^3 step ({dt:.1f} s), FP64 C restatement of the reference algorithm "
                      "(OpenMP), GMRES(30) to 1e-12"}


# ------------------------------------------------------------------ thermal initial condition
THERMAL_BETA = 10.0
# algorithmic bytes per site of one Gauss projection sweep: k_gauss_g reads E
# (192 B) and the links (432 B) and writes G (144 B); k_gauss_sweep reads G,
# E and the links and writes E (144 + 192 + 432 + 192 B)
THERMAL_BYTES_SITE_SWEEP = 768 + 960


def measure_thermal_ic(L, seed=1, cpu=True, cpu_sweeps=4, max_sweeps=200000):
    """EquilibriumInit (beta 10, one round, no leapfrog steps) on an L^3
    lattice of the open module context.  Timed apart, with CUDA events on the
    context's stream: the round without projection (cold links, the host
    ranlxd draw of the thermal field, its upload) and the Gauss projection of
    that field to 1e-3 (the device part, and the bulk of the work).  The CPU
    leg times `cpu_sweeps` sweeps of the oracle's projection on the same
    drawn field."""
    import torch
    from nrqcd_b200 import GaugeConfiguration, _capi, lattice
    ctx = lattice.context()
    stream = torch.cuda.ExternalStream(_capi.load().nrq_cuda_stream(ctx))
    g = GaugeConfiguration()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    draw = lambda: g.EquilibriumInit(THERMAL_BETA, 1, 0, tolerance_Eprojection=1e30,  # noqa: E731
                                     RandomSeed=seed, verbose=False)
    draw()  # warm-up: allocations
    g.GaussProjection(1e-3, max_sweeps=max_sweeps)
    _, draw_ms = timed(draw)
    (sweeps, dev), ms = timed(lambda: g.GaussProjection(1e-3, max_sweeps=max_sweeps))
    del g
    V = L ** 3
    out = {"config": {"lattice": [L, L, L], "beta": THERMAL_BETA, "nefieldinit": 1, "nequilibrium": 0,
                      "tolerance": 1e-3, "seed": seed},
           "sweeps": int(sweeps), "final_deviation": float(dev), "projection_ms": ms,
           "ms_per_sweep": ms / max(1, sweeps),
           "site_sweeps_per_s": V * sweeps / (ms / 1000.0),
           "algorithmic_bytes_per_site_sweep": THERMAL_BYTES_SITE_SWEEP,
           "algorithmic_GBps": THERMAL_BYTES_SITE_SWEEP * V * sweeps / (ms / 1000.0) / 1e9,
           "draw_ms": draw_ms,
           "draw_note": "cold links and the device ranlxd draw of the thermal field: the reference's one "
                        "stream, each device thread from a starting state the host jumps to (one modular "
                        "multiplication per state), written into the field's planes"}
    if cpu:
        from oracle import oracle as oc
        n = (L, L, L)
        links, ef, _, _, _ = oc.equilibrium_init(n, A, THERMAL_BETA, 1, 0, tol=1e30, seed=seed)
        t0 = time.perf_counter()
        done = oc.gauss_project(n, A, links, ef, tol=1e-3, max_sweeps=cpu_sweeps)
        dt = time.perf_counter() - t0
        cps = V * done / dt
        out["cpu_baseline"] = {"value": cps, "unit": "site-sweeps/s", "cores": oc.num_threads(), "kind": "port",
                               "sample": f"{done} projection sweeps of the oracle at {L}^3 ({dt:.2f} s)"}
        out["speedup_vs_cpu"] = out["site_sweeps_per_s"] / cps
    return out


# ------------------------------------------------------------------ gluon distribution
# algorithmic bytes per site of one Coulomb gauge-fixing iteration outside the
# FFTs: divergence (links 432 read, D 144 written), acceleration (D read and
# written), exponential (D read and written), transformation (D 144, links
# 432 read and written)
GF_BYTES_SITE_ITER = (432 + 144) + 288 + 288 + (144 + 864)


def measure_gluon_distribution(L, cpu=True, steps=10):
    """Coulomb gauge fixing (tolerance 1e-8, alpha 0.08, at most 100
    iterations) and the transverse AA/EE correlators of an L^3 box initial
    condition (aQ = 0.5, n0 = 1, seed 1, random links) after `steps` leapfrog
    steps, timed with CUDA events on the context's stream; the CPU leg times
    two iterations and the correlators of the oracle on the same links."""
    import torch
    from nrqcd_b200 import GaugeConfiguration, _capi, lattice
    ctx = lattice.context()
    stream = torch.cuda.ExternalStream(_capi.load().nrq_cuda_stream(ctx))
    g = GaugeConfiguration()
    g.TransversePolarisedOccupiedInit_Box(0.5, 1.0, 0.0, RandomSeed=1, identity_links=False)
    for _ in range(steps):
        g.Update(1.0)
    links, ef = g.download()
    w = GaugeConfiguration()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        e1.synchronize()
        return r, e0.elapsed_time(e1)

    w.assign(g)
    w.CoulombGaugefixing(1e-8, 0.08, 100, verbose=False)  # warm-up (cuFFT plans, allocations)
    w.GetTransverseCorrelators()
    w.assign(g)
    (it, dev), gf_ms = timed(lambda: w.CoulombGaugefixing(1e-8, 0.08, 100, verbose=False))
    _, corr_ms = timed(w.GetTransverseCorrelators)
    del w, g
    V = L ** 3
    transforms = int(min(it, 100)) - (1 if it <= 100 else 0)
    out = {"config": {"lattice": [L, L, L], "initial_condition": "box aQ=0.5 n0=1 seed 1, random links",
                      "leapfrog_steps": steps, "tolerance": 1e-8, "alpha": 0.08, "max_iterations": 100},
           "gaugefix_loop_counter": int(it), "gauge_transformations": transforms,
           "final_divergence": float(dev[-1]), "gaugefix_ms": gf_ms,
           "gaugefix_ms_per_transformation": gf_ms / max(1, transforms),
           "gaugefix_nonfft_bytes_per_site_iteration": GF_BYTES_SITE_ITER,
           "correlators_ms": corr_ms,
           "note": "per gauge-fixing iteration: divergence + its max, 9 forward and 9 inverse cuFFT Z2Z, "
                   "acceleration, exponential, transformation; correlators: algebra coordinates (Jacobi "
                   "ArgLogU), 48 forward cuFFT Z2Z, projection"}
    if cpu:
        from oracle import oracle as oc
        n = (L, L, L)
        l2 = links.copy()
        t0 = time.perf_counter()
        oc.coulomb_gaugefix(n, A, l2, tol=0.0, alpha=0.08, max_iterations=2)
        t_gf = (time.perf_counter() - t0) / 2
        t0 = time.perf_counter()
        oc.transverse_correlators(n, A, links, ef)
        t_corr = time.perf_counter() - t0
        out["cpu_baseline"] = {"gaugefix_ms_per_transformation": t_gf * 1e3, "correlators_ms": t_corr * 1e3,
                               "cores": oc.num_threads(), "kind": "port",
                               "sample": f"2 gauge-fixing iterations and one correlator pass of the oracle at {L}^3"}
        out["speedup_vs_cpu"] = {"gaugefix": t_gf * 1e3 / out["gaugefix_ms_per_transformation"],
                                 "correlators": t_corr * 1e3 / corr_ms}
    return out


# ------------------------------------------------------------------ CN forms
# name -> (form, history start, merged update, confirm every solve) of the
# plain form; the speed-ups are against plain_fp64_bicgstab, the library's
# default plain solve (start extrapolated from the field's history, x, r and
# p updated in one pass, the recursive residual accepted with the measured
# margin); beside it the plain solve from 2b - psi alone and the plain solve
# with two update passes and every solve confirmed by the true residual
FORMS = {"plain_fp64_bicgstab": (0, 1, 1, 0), "plain_fp64_bicgstab_no_history": (0, 0, 1, 0),
         "plain_fp64_bicgstab_two_pass_confirmed": (0, 1, 0, 1),
         "precision_fp32_chebyshev_fp64_refinement": (1, 1, 1, 0), "learned_guess_precision": (2, 1, 1, 0)}
FORMS_SIZES = (64, 96, 128)
# lattices of the precision form's drift (the precision configuration names 64^3 and 96^3)
DRIFT_SIZES = (64, 96)


def train_learned(tol=1e-10, masses=(MASS,)):
    """The learned form's network, trained on seeded 32^3 solves (2
    configurations x the given heavy masses x 8 steps); the parameters load
    into any lattice size.  The FP32 output bias is per species and history
    depth, not per mass, so a network serves best at the masses it was
    trained on: the forms use aM = 1.0, the ensemble aM = 1.0 and 1.5."""
    from nrqcd_b200.learned import train_on_seeded_configs
    t0 = time.perf_counter()
    params, info = train_on_seeded_configs(extent=32, configs=(11, 12), steps=8, masses=tuple(masses),
                                           WilsonCoeffs=WILSON, spacings=A, tol=tol,
                                           iterations=800 if len(masses) == 1 else 1000)
    info["wall_s"] = time.perf_counter() - t0
    return params, info


def measure_cn_forms(L, steps, params, tol=1e-10, seed=1):
    """CN-only seconds per step of every solver form at the same residual on
    one L^3 gauge field (the headline's comparison at <= 1e-10): a fresh point
    source per form, 3 warm-up and `steps` timed CN steps, CUDA events on the
    lattice's stream."""
    import torch
    from nrqcd_b200 import GaugeConfiguration, NRQCDField, _capi, lattice
    from nrqcd_b200.learned import LearnedGuess
    lib = _capi.load()
    lat = lattice.Lattice((L, L, L), A)
    out = {}
    try:
        g = GaugeConfiguration(lat=lat)
        g.TransversePolarisedOccupiedInit_Box(0.5, 1.0, 0.0, RandomSeed=seed, identity_links=True)
        stream = torch.cuda.ExternalStream(lib.nrq_cuda_stream(lat.ctx))
        cw = _capi.coeffs(WILSON)
        for name, (form, hist, merged, confirm) in FORMS.items():
            cn = ctypes.c_void_p()
            _capi.check(lib.nrq_cn_init(lat.ctx, MASS, _capi.dptr(cw), 1.0, tol, 10000, form, ctypes.byref(cn)),
                        lat.ctx, "nrq_cn_init")
            _capi.check(lib.nrq_cn_set_history_guess(cn, hist), lat.ctx, "history guess")
            _capi.check(lib.nrq_cn_set_merged_update(cn, merged), lat.ctx, "merged update")
            _capi.check(lib.nrq_cn_set_true_residual(cn, confirm), lat.ctx, "true residual")
            net = None
            if form == 2:
                net = LearnedGuess(lat=lat)
                net.params = params
                net.set_trained(True)
                net.attach(cn)
            h = NRQCDField(lat=lat)
            h.InitSinglePoint(1, 1)

            def update():
                st = _capi.CnStats()
                _capi.check(lib.nrq_heavy_update_cn(cn, h.handle, g.handle, MASS, _capi.dptr(cw), 1.0,
                                                    ctypes.byref(st)), lat.ctx, "update")
                return st.as_dict()
            for _ in range(3):
                update()
            stats = []
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(steps):
                stats.append(update())
            e1.record(stream)
            e1.synchronize()
            ms = e0.elapsed_time(e1) / steps
            which = ctypes.c_int()
            tune = np.zeros(4)
            _capi.check(lib.nrq_cn_stencil_info(cn, ctypes.byref(which), _capi.dptr(tune)), lat.ctx, "stencil_info")
            out[name] = {"s_per_step": ms / 1000.0, "tol": tol,
                         "max_rel_residual": max(st["max_rel_residual"] for st in stats),
                         "fp64_stencil": STENCIL_NAMES[which.value],
                         "fp64_stencil_tuning_ms": [float(t) for t in tune],
                         "stencil_launches_per_step": float(np.mean([st["matvecs"] for st in stats])),
                         "inner_steps_per_step": float(np.mean([st["iterations"] for st in stats])),
                         "initial_rel_residual": float(np.mean([st["initial_rel_residual"] for st in stats])),
                         "norms": [h.GetNorm_Quark(), h.GetNorm_AntiQ()]}
            if net is not None:
                net.detach(cn)
                net.Destructor()
            h.Destructor()
            lib.nrq_cn_finalize(cn)
        g.Deallocate()
    finally:
        lat.close()
    base = out["plain_fp64_bicgstab"]["s_per_step"]
    for v in out.values():
        v["speedup_vs_plain_fp64"] = base / v["s_per_step"]
    return out


def measure_all_forms(steps, sizes=FORMS_SIZES, learned=None):
    params, info = train_learned() if learned is None else learned
    res = {"learned_training": info}
    for L in sizes:
        res[f"{L}^3"] = measure_cn_forms(L, steps, params)
    return res


# ------------------------------------------------------------------ precision drift
def measure_precision_drift(L, n0, steps, seed=1):
    """The precision form end to end (FP32-link leapfrog with FP64
    reunitarisation every 10 steps, FP32 Chebyshev CN with FP64 refinement
    at 1e-10), its CN half alone on FP64 links, and the FP64 path at 1e-10,
    against the FP64 path (FP64 leapfrog, plain FP64 CN at 1e-12) from the
    same seeded fields: the drift of every observable after `steps` coupled
    steps, and the s/step of every path (CUDA events)."""
    import torch
    from nrqcd_b200 import GaugeConfiguration, NRQCDField, _capi, lattice
    lib = _capi.load()
    lat = lattice.Lattice((L, L, L), A)
    cw = _capi.coeffs(WILSON)
    out = {"lattice": [L, L, L], "n0": n0, "steps": steps}
    try:
        stream = torch.cuda.ExternalStream(lib.nrq_cuda_stream(lat.ctx))
        paths = {}
        # the FP64 path at the headline residual (the drift reference), the
        # FP64 path at the forms' residual 1e-10, the whole precision form
        # (FP32-link leapfrog and FP32 Chebyshev CN with FP64 refinement), and
        # its CN half alone on FP64 links
        for name, form, tol, prec in (("fp64", 0, 1e-12, 0), ("fp64_1e-10", 0, 1e-10, 0),
                                      ("precision", 1, 1e-10, 1), ("precision_cn_fp64_links", 1, 1e-10, 0)):
            g = GaugeConfiguration(lat=lat)
            g.TransversePolarisedOccupiedInit_Box(0.5, n0, 0.0, RandomSeed=seed, identity_links=True)
            if prec:
                g.SetPrecision(1, 10)
            h = NRQCDField(lat=lat)
            h.InitSinglePoint(1, 1)
            cn = ctypes.c_void_p()
            _capi.check(lib.nrq_cn_init(lat.ctx, MASS, _capi.dptr(cw), 1.0, tol, 10000, form, ctypes.byref(cn)),
                        lat.ctx, "nrq_cn_init")
            e_start = g.GetEnergy()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            its, mvs = [], []
            for _ in range(steps):
                st = _capi.CnStats()
                _capi.check(lib.nrq_heavy_update_cn(cn, h.handle, g.handle, MASS, _capi.dptr(cw), 1.0,
                                                    ctypes.byref(st)), lat.ctx, "update")
                its.append(st.iterations)
                mvs.append(st.matvecs)
                g.Update(1.0)
            e1.record(stream)
            e1.synchronize()
            which = ctypes.c_int()
            _capi.check(lib.nrq_cn_stencil_info(cn, ctypes.byref(which), None), lat.ctx, "stencil_info")
            paths[name] = {"g": g, "h": h, "cn": cn, "ms": e0.elapsed_time(e1) / steps, "e_start": e_start,
                           "solve": {"fp64_stencil": STENCIL_NAMES[which.value],
                                     "iterations_per_step": float(np.mean(its)),
                                     "stencil_launches_per_step": float(np.mean(mvs))}}
        res = {}
        for name, p in paths.items():
            g, h = p["g"], p["h"]
            en = g.GetEnergy()
            gref, gmax = g._gauss()
            res[name] = {"s_per_step": p["ms"] / 1000.0, **p["solve"], "energy": en,
                         "energy_drift_rel": abs(en - p["e_start"]) / abs(p["e_start"]),
                         "gauss_max_norm": gmax, "norm_quark_minus_1": h.GetNorm_Quark() - 1.0,
                         "norm_antiq_minus_1": h.GetNorm_AntiQ() - 1.0,
                         "unitarity_max_dev": g.GetUnitarityDeviation()[0]}
        la, ea = paths["fp64"]["g"].download()
        qa, aa = paths["fp64"]["h"].download()

        def drift(name):
            lb, eb = paths[name]["g"].download()
            qb, ab = paths[name]["h"].download()
            r, f = res[name], res["fp64"]
            return {"energy_rel": abs(r["energy"] - f["energy"]) / abs(f["energy"]),
                    "gauss_max_norm_abs": abs(r["gauss_max_norm"] - f["gauss_max_norm"]),
                    "links_max_abs": float(np.abs(lb - la).max()), "efield_max_abs": float(np.abs(eb - ea).max()),
                    "propagator_max_abs": float(max(np.abs(qb - qa).max(), np.abs(ab - aa).max())),
                    "norm_abs": abs(r["norm_quark_minus_1"] - f["norm_quark_minus_1"])}
        for name in res:
            out[name] = res[name]
        out["drift_vs_fp64"] = drift("precision")
        out["drift_vs_fp64_by_path"] = {name: drift(name) for name in res if name != "fp64"}
        out["speedup_coupled_step"] = res["fp64"]["s_per_step"] / res["precision"]["s_per_step"]
        out["speedup_vs_fp64_at_1e-10"] = {name: res["fp64_1e-10"]["s_per_step"] / res[name]["s_per_step"]
                                           for name in ("precision", "precision_cn_fp64_links")}
        for p in paths.values():
            lib.nrq_cn_finalize(p["cn"])
            p["h"].Destructor()
            p["g"].Deallocate()
    finally:
        lat.close()
    return out


# ------------------------------------------------------------------ batching ensemble
# 8 members at 24^3, 4 at 32^3, 2 at 48^3; 16 point sources at random sites x
# masses aM = 1.0 and 1.5 per member; precision-form CN at residual 1e-10
ENSEMBLE = ((24, 8), (32, 4), (48, 2))
ENS_SOURCES = 16
ENS_MASSES = (1.0, 1.5)


def measure_ensemble(steps, warmup, tol=1e-10, learned_params=None, ensemble=ENSEMBLE, sources=ENS_SOURCES):
    """Aggregate field-site updates/s of the uneven ensemble: one CUDA graph
    launch per coupled step, the same batched launches issued eagerly, and a
    serial loop of single-field precision-form updates (nrq_heavy_update_cn
    per field, then the leapfrog per member).  ensemble: (extent, members)
    pairs; sources: point sources per member and mass."""
    import torch
    from nrqcd_b200 import GaugeConfiguration, NRQCDField, _capi, lattice
    from nrqcd_b200.batch import CNBatch, Ensemble
    lib = _capi.load()
    lats = {L: lattice.Lattice((L, L, L), A) for L, _ in ensemble}
    members = []
    seed = 1000
    for L, count in ensemble:
        for _ in range(count):
            seed += 1
            g = GaugeConfiguration(lat=lats[L])
            g.TransversePolarisedOccupiedInit_Box(0.5, 1.0, 0.0, RandomSeed=seed, identity_links=True)
            rng = np.random.default_rng(seed)
            srcs = rng.integers(0, L ** 3, size=(sources, 2)) + 1
            fields, masses = [], []
            for m in ENS_MASSES:
                for lq, la in srcs:
                    h = NRQCDField(lat=lats[L])
                    h.InitSinglePoint(int(lq), int(la))
                    fields.append(h)
                    masses.append(m)
            members.append((L, g, fields, masses))
    per_step = sum(L ** 3 * len(f) for L, _, f, _ in members)
    streams = [torch.cuda.ExternalStream(lib.nrq_cuda_stream(lats[L].ctx)) for L, _ in ensemble]
    s0 = streams[0]

    def timed(fn, n):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        for _ in range(n):
            fn()
        for s in streams[1:]:
            s0.wait_stream(s)
        e1.record(s0)
        e1.synchronize()
        return e0.elapsed_time(e1) / n / 1000.0

    batches = [CNBatch(f, m, tol, lat=lats[L]) for L, _, f, m in members]
    ens = Ensemble(batches, [g for _, g, _, _ in members])
    stats = []
    # the fields' history fills (depth 0 to 4, a calibration at each), then
    # the graph capture
    for _ in range(max(6, warmup)):
        ens.Step(WILSON, 1.0, use_graph=True)
    t_graph = timed(lambda: stats.append(ens.Step(WILSON, 1.0, use_graph=True)), steps)
    # the same batched launches without the graph, with per-class kernel timing
    for L in lats:
        _capi.profile_enable(lats[L].ctx, True)
    t_eager = timed(lambda: stats.append(ens.Step(WILSON, 1.0, use_graph=False)), steps)
    prof = {L: _capi.profile_read(lats[L].ctx) for L in lats}
    for L in lats:
        _capi.profile_enable(lats[L].ctx, False)
    info = {L: b.info() for (L, _, _, _), b in zip(members, batches)}
    # forms combined: every batch starts its solves from the learned guess
    t_learned, info_learned, learned_stats, gates_learned = None, None, [], None
    if learned_params is not None:
        from nrqcd_b200.learned import LearnedGuess
        nets = {}
        for L in lats:
            nets[L] = LearnedGuess(lat=lats[L])
            nets[L].params = learned_params
            nets[L].set_trained(True)
        for (L, _, _, _), b in zip(members, batches):
            b.attach_learned(nets[L])
        # history fills (depth 0, 1, 2), the gate decides at depth 2, then
        # calibration (with the guess or, gated off, without) and capture
        for _ in range(max(6, warmup + 3)):
            ens.Step(WILSON, 1.0, use_graph=True)
        t_learned = timed(lambda: learned_stats.append(ens.Step(WILSON, 1.0, use_graph=True)), steps)
        info_learned = {L: b.info() for (L, _, _, _), b in zip(members, batches)}
        gates_learned = {}
        for (L, _, _, _), b in zip(members, batches):
            gi = b.learned_info()
            gates_learned.setdefault(f"{L}^3", []).append(
                {"gate": gi["gate"], "guess_ms": round(gi["guess_ms"], 3), "saving_ms": round(gi["saving_ms"], 3)})
        for b in batches:
            b.attach_learned(None)
        for net in nets.values():
            net.Destructor()
    ens.Destructor()
    for b in batches:
        b.Destructor()
    # serial loop of single-field updates (precision form, same tolerance)
    cns = {}
    for L in lats:
        h = ctypes.c_void_p()
        _capi.check(lib.nrq_cn_init(lats[L].ctx, ENS_MASSES[0], _capi.dptr(_capi.coeffs(WILSON)), 1.0, tol, 10000, 1,
                                    ctypes.byref(h)), lats[L].ctx, "nrq_cn_init")
        cns[L] = h
    cw = _capi.coeffs(WILSON)
    serial_stats = []

    def serial_step():
        for L, g, fields, masses in members:
            for h, m in zip(fields, masses):
                st = _capi.CnStats()
                _capi.check(lib.nrq_heavy_update_cn(cns[L], h.handle, g.handle, m, _capi.dptr(cw), 1.0,
                                                    ctypes.byref(st)), lats[L].ctx, "serial update")
                serial_stats.append(st.max_rel_residual)
            g.Update(1.0)

    serial_step()  # warm-up
    serial_steps = max(1, min(steps, 2))
    t_serial = timed(serial_step, serial_steps)
    for L in lats:
        lib.nrq_cn_finalize(cns[L])
    sten = {}
    for L in lats:
        c0 = prof[L]["cn_stencil"]
        sten[f"{L}^3"] = {"launches": c0["launches"], "ms": c0["ms"],
                          "achieved_GBps": c0["bytes"] / (c0["ms"] / 1000.0) / 1e9 if c0["ms"] > 0 else None}
    out = {
        "workload": "uneven ensemble " + " + ".join(f"{n} x {L}^3" for L, n in ensemble) +
                    f", {sources} point sources at random sites x aM = 1.0, "
                    "1.5 per member, coupled step (CN of every field, then the member's leapfrog), "
                    "precision-form CN at residual 1e-10",
        "field_site_updates_per_step": per_step,
        "graph": {"s_per_step": t_graph, "field_site_updates_per_s": per_step / t_graph},
        "eager_batched": {"s_per_step": t_eager, "field_site_updates_per_s": per_step / t_eager,
                          "stencil_kernels": sten},
        "serial_single_field": {"s_per_step": t_serial, "field_site_updates_per_s": per_step / t_serial,
                                "steps": serial_steps, "max_rel_residual": max(serial_stats)},
        "speedup_graph_vs_serial": t_serial / t_graph,
        "graph_learned_guess": None if t_learned is None else {
            "s_per_step": t_learned, "field_site_updates_per_s": per_step / t_learned,
            "speedup_vs_serial": t_serial / t_learned,
            "max_rel_residual": max(st["max_rel_residual"] for st in learned_stats),
            "schedules": {f"{L}^3": v["schedule"] for L, v in info_learned.items()},
            "gates": gates_learned},
        "max_rel_residual": max(s["max_rel_residual"] for s in stats),
        "converged": all(s["converged"] == 1 for s in stats),
        "tuning": {f"{L}^3": v for L, v in info.items()},
    }
    for _, g, fields, _ in members:
        for h in fields:
            h.Destructor()
        g.Deallocate()
    for L in lats:
        lats[L].close()
    return out


# ------------------------------------------------------------------ our arm
def measure_fp64_peak(n=8192, reps=5):
    """FP64 arithmetic peak of this GPU for the compute side of the stencil's
    roofline: a cuBLAS DGEMM (torch.matmul, float64) of n^3, best of `reps`,
    CUDA events; measured after the timed region."""
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best / 1000.0) / 1e12


def leapfrog_summary(ms_per_step, prof, V, peak_gbps, fp64_tflops):
    """Leapfrog-only steps: site-updates/s, and the force kernel against the
    HBM and FP64 rooflines (its 816 B and 5,832 flops per site put it above
    the FP64 ridge, so the FP64 peak bounds it)."""
    ef, lk = prof["leapfrog_efield"], prof["leapfrog_links"]
    ef_ms = ef["ms"] / max(1, ef["launches"])
    out = {"ms_per_step": ms_per_step, "site_updates_per_s": V / (ms_per_step / 1000.0),
           "links_ms": lk["ms"] / max(1, lk["launches"]), "force_ms": ef_ms}
    if ef_ms > 0:
        gbps = ef["bytes"] / max(1, ef["launches"]) / (ef_ms / 1000.0) / 1e9
        tf = LEAPFROG_FORCE_FLOPS_PER_SITE * V / (ef_ms / 1000.0) / 1e12
        out["force"] = {"algorithmic_GBps": gbps, "hbm_frac": gbps / peak_gbps, "fp64_tflops": tf,
                        "fp64_frac": tf / fp64_tflops, "flops_per_site": LEAPFROG_FORCE_FLOPS_PER_SITE,
                        "bytes_per_site": 816}
    return out


def member_seed(rank):
    """ranlxd seed of the ensemble member a rank evolves (replicas)."""
    return 1 + rank


def timed_steps(step, steps, dist, timer):
    """The timed region of every rank: a barrier, `steps` calls of step()
    between timer.start() and timer.stop() (milliseconds), a barrier, and the
    max of the durations over the ranks."""
    if dist is not None:
        dist.barrier()
    timer.start()
    for _ in range(steps):
        step()
    ms = timer.stop()
    if dist is not None:
        dist.barrier()
    return max_over_ranks(ms, dist)


def whole_job_rate(world, sites, steps, ms):
    """Site-updates per second of the whole job: every rank's lattice
    advanced `steps` times within the slowest rank's `ms`."""
    return world * sites * steps / (ms / 1000.0)


class CudaEventTimer:
    """Device time on `stream` between start() and stop() (milliseconds)."""

    def __init__(self, stream):
        import torch
        self.torch = torch
        self.stream = stream

    def start(self):
        self.torch.cuda.synchronize()
        self.e0 = self.torch.cuda.Event(enable_timing=True)
        self.e1 = self.torch.cuda.Event(enable_timing=True)
        self.e0.record(self.stream)

    def stop(self):
        self.e1.record(self.stream)
        self.e1.synchronize()
        self.torch.cuda.synchronize()
        return self.e0.elapsed_time(self.e1)


def max_over_ranks(x, dist=None):
    """Max of a per-rank float over all ranks (the timed region's duration);
    identity without a process group.  NCCL reduces a CUDA tensor, gloo a
    CPU one."""
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def free_port():
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def relaunch_ranks(n):
    """`--gpus N` without a launcher: start the N ranks with
    torch.distributed.run on this node (rendezvous on 127.0.0.1) and return
    its exit status; rank 0's JSON line passes through."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(free_port()), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(relaunch_ranks(args.gpus))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        raise SystemExit(f"bench.py: --gpus {args.gpus} but the launcher started {world} ranks")
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist_
        import datetime
        dist = dist_
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    if args.impl == "reference":
        run_reference(args, rank)
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.only_drift:
        import torch
        torch.cuda.set_device(local)
        out = [measure_precision_drift(size, n0, 20) for size in DRIFT_SIZES for n0 in (0.5, 1.0, 2.0)]
        if rank == 0:
            print(json.dumps({"precision_drift": out}), flush=True)
        return
    if args.only_ensemble:
        import torch
        torch.cuda.set_device(local)
        ens = ENSEMBLE
        if args.ensemble_members:
            ens = tuple((int(a), int(b)) for a, b in (m.split("x") for m in args.ensemble_members.split(",")))
        learned = None if args.ensemble_no_learned else train_learned(masses=ENS_MASSES)[0]
        out = measure_ensemble(args.steps, args.warmup, learned_params=learned, ensemble=ens,
                               sources=args.ensemble_sources or ENS_SOURCES)
        if rank == 0:
            print(json.dumps({"batching_ensemble": out}), flush=True)
        return

    import torch
    from nrqcd_b200 import GaugeConfiguration, NRQCDField, _capi, lattice, nrqcd

    L = args.size
    V = L ** 3
    torch.cuda.set_device(local)
    lattice.InitModule([L, L, L], list(A), device=local)
    ctx = lattice.context()
    nrqcd.InitModule(MASS, WILSON, 1.0, TOL)
    if args.stencil != "timed":
        nrqcd.SetStencil({"register": nrqcd.STENCIL_REGISTER, "tma": nrqcd.STENCIL_TMA,
                          "tensor": nrqcd.STENCIL_TENSOR, "fma": nrqcd.STENCIL_FMA}[args.stencil])
    if args.two_pass:
        nrqcd.SetMergedUpdate(False)
    if args.history_depth is not None:
        nrqcd.SetHistoryDepth(args.history_depth)
    g = GaugeConfiguration()
    g.TransversePolarisedOccupiedInit_Box(0.5, 1.0, 0.0, RandomSeed=member_seed(rank), identity_links=True)
    h = NRQCDField()
    h.InitSinglePoint(1, 1)
    lib = _capi.load()
    stream = torch.cuda.ExternalStream(lib.nrq_cuda_stream(ctx))
    if args.only_gluon:
        out = measure_gluon_distribution(L, cpu=not args.no_cpu_baseline)
        if rank == 0:
            print(json.dumps({"gluon_distribution": out}), flush=True)
        del h, g
        nrqcd.FinalizeModule()
        lattice.FinalizeModule()
        return
    if args.only_thermal:
        out = measure_thermal_ic(L, cpu=not args.no_cpu_baseline)
        if rank == 0:
            print(json.dumps({"thermal_initial_condition": out}), flush=True)
        del h, g
        nrqcd.FinalizeModule()
        lattice.FinalizeModule()
        return
    if args.only_forms:
        forms = measure_all_forms(max(2, min(args.steps, 5)), sizes=tuple(args.forms_sizes))
        if rank == 0:
            print(json.dumps({"cn_forms_at_1e-10": forms}), flush=True)
        del h, g
        nrqcd.FinalizeModule()
        lattice.FinalizeModule()
        return

    iters = []

    def step():
        st = h.Update(g, MASS, WILSON, 1.0)
        iters.append(st)
        g.Update(1.0)

    clocks = ClockSampler(local)
    clocks.start()
    for _ in range(max(3, args.warmup)):
        step()
    lattice.synchronize()
    iters.clear()
    # ---------------- timed region
    torch.cuda.synchronize()
    clocks.mark()
    _capi.profile_enable(ctx, True)
    ms = timed_steps(step, args.steps, dist, CudaEventTimer(stream))
    prof = _capi.profile_read(ctx)
    _capi.profile_enable(ctx, False)
    clk = clocks.stop()
    ms_per_step = ms / args.steps
    value = whole_job_rate(world, V, args.steps, ms)
    norm_q, norm_a = h.GetNorm_Quark(), h.GetNorm_AntiQ()
    which, tune_ms = nrqcd.StencilInfo()
    p64 = measure_fp64_peak()
    stencil = {"in_use": nrqcd.STENCIL_NAMES[which],
               "tuning_ms_per_launch": {"k_cn_mv2": float(tune_ms[0]), "k_cn_mv3_with_vec_s": float(tune_ms[1]),
                                        "k_cn_mv4_with_vec_s": float(tune_ms[2]),
                                        "k_cn_mv5_with_vec_s": float(tune_ms[3])}}

    # ---------------- leapfrog-only steps (the long leapfrog phases before the
    # propagators start), CUDA events on the library stream
    lf_steps = 50
    _capi.profile_enable(ctx, True)
    lf_ms = timed_steps(lambda: g.Update(1.0), lf_steps, dist, CudaEventTimer(stream)) / lf_steps
    lf_prof = _capi.profile_read(ctx)
    _capi.profile_enable(ctx, False)

    # ---------------- end-to-end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True)  # noqa: E731
        links_h = pin((V, 3, 3, 3, 2), torch.float64)
        ef_h = pin((V, 3, 8), torch.float64)
        q_h = pin((V, 6, 6, 2), torch.float64)
        a_h = pin((V, 6, 6, 2), torch.float64)
        P = lambda t: ctypes.cast(t.data_ptr(), _capi._dp)  # noqa: E731
        _capi.check(lib.nrq_gauge_download(g.handle, P(links_h), P(ef_h)), ctx, "download")
        _capi.check(lib.nrq_heavy_download(h.handle, P(q_h), P(a_h)), ctx, "download")
        e2e_steps = max(1, min(args.steps, 5))
        h2d = (links_h.numel() + ef_h.numel() + q_h.numel() + a_h.numel()) * 8
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if dist is not None:
            dist.barrier()
        e0.record(stream)
        for _ in range(e2e_steps):
            _capi.check(lib.nrq_gauge_upload(g.handle, P(links_h), P(ef_h)), ctx, "upload")
            _capi.check(lib.nrq_heavy_upload(h.handle, P(q_h), P(a_h)), ctx, "upload")
            step()
            _capi.check(lib.nrq_heavy_download(h.handle, P(q_h), P(a_h)), ctx, "download")
            _capi.check(lib.nrq_gauge_download(g.handle, P(links_h), P(ef_h)), ctx, "download")
        e1.record(stream)
        e1.synchronize()
        ems = max_over_ranks(e0.elapsed_time(e1), dist)
        e2e = {"value": world * V * e2e_steps / (ems / 1000.0), "unit": "site-updates/s",
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(h2d), "steps": e2e_steps,
               "path": "nrq_gauge_upload + nrq_heavy_upload + nrq_heavy_update_cn + nrq_gauge_update + "
                       "nrq_heavy_download + nrq_gauge_download, pinned host buffers"}

    # the host-synchronised loops of the gluon observables and the thermal
    # initial condition run first, before the ensemble's and the forms' state
    # fills the device
    gluon = None
    if not args.no_gluon and world == 1:
        gluon = measure_gluon_distribution(L, cpu=not args.no_cpu_baseline)

    thermal = None
    if not args.no_thermal and world == 1:
        thermal = measure_thermal_ic(L, cpu=not args.no_cpu_baseline)

    ensemble = None
    if not args.no_ensemble and world == 1:
        ensemble = measure_ensemble(max(2, min(args.steps, 3)), 2,
                                    learned_params=train_learned(masses=ENS_MASSES)[0])

    drift = None
    if not args.no_drift and world == 1:
        drift = [measure_precision_drift(size, n0, 20) for size in DRIFT_SIZES for n0 in (0.5, 1.0, 2.0)]

    forms = None
    if not args.no_forms and world == 1:
        forms = measure_all_forms(max(2, min(args.steps, 5)), sizes=tuple(args.forms_sizes))

    if rank == 0:
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        peak, peak_src = 6650.0, "fallback"
        if os.path.exists(peaks_path):
            peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
        sten = prof["cn_stencil"]
        # the library's stencil class counts the byte model's bytes of a
        # 12-column launch: U and E once per species (2 x 624 B) plus 1152 B
        # per vector stream; the tensor-core stencil's design reads its cached
        # 6x6 blocks (3456 B) and diagonal matrices (216 B) in place of U and
        # E, reported beside it and not credited
        achieved = sten["bytes"] / (sten["ms"] / 1000.0) / 1e9 if sten["ms"] > 0 else None
        tensor = which in (nrqcd.STENCIL_TENSOR, nrqcd.STENCIL_FMA)
        blk_bytes = 3552.0 if which == nrqcd.STENCIL_FMA else 3456.0
        design_bytes = sten["bytes"] + (sten["launches"] * V * (blk_bytes + 216.0 - 1248.0) if tensor else 0.0)
        # FP64 arithmetic of one 12-column stencil launch per site: 2 species x
        # (6 neighbours x 6 columns x 36 + 6 columns x 18) complex FMAs (4 DFMA
        # each, 2 flops per DFMA) plus the block assembly (~270 complex FMAs)
        # (the tensor-core stencil reads the blocks assembled once per update,
        # and its MMA tiles carry 16/12 x 8/6 of these products with padding)
        flops_site = 2 * (6 * 6 * 36 + 6 * 18 + (0 if tensor else 270)) * 4 * 2
        fp64_achieved = flops_site * V * sten["launches"] / (sten["ms"] / 1000.0) / 1e12 if sten["ms"] > 0 else None
        step_bytes = sum(v["bytes"] for v in prof.values()) / args.steps
        # the build plan's per-site byte model of a coupled step: leapfrog
        # 1872 B; per species and 6-column matvec 1776 B (spinor in and out,
        # U and E, derived blocks not credited) and per 6-column vector
        # stream 576 B, with the matvecs and streams the solves executed
        mv = float(np.mean([st["matvecs"] for st in iters])) if iters else 0.0
        vs = float(np.mean([st["vector_streams"] for st in iters])) if iters else 0.0
        model_site = 1872.0 + 2 * (mv * 1776.0 + vs * 576.0)
        model_gbps = model_site * V / (ms_per_step / 1000.0) / 1e9
        model = {"bytes_per_site_step": model_site, "matvecs_per_step": mv, "vector_streams_per_step": vs,
                 "GBps": model_gbps, "frac": model_gbps / peak, "peak_source": peak_src}
        its = [s["iterations"] for s in iters]
        line = {
            "metric": METRIC, "value": value, "unit": "site-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(L, world),
                           bicgstab_update="two-pass" if args.two_pass else "merged",
                           history_depth=args.history_depth if args.history_depth is not None else "default"),
            "roofline": {"bound": "hbm", "kernel": "CN 12-column stencil: " + stencil["in_use"],
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_source": peak_src,
                         "traffic": (STENCIL_DRAM_BYTES_PER_SITE[which] * V / 1e9
                                     if which in STENCIL_DRAM_BYTES_PER_SITE else None),
                         "traffic_unit": "GB per launch (ncu capture of one 64^3 update, per site x V)",
                         "algorithmic_GB_per_launch": sten["bytes"] / max(1, sten["launches"]) / 1e9,
                         "algorithmic_bytes": "per 12-column launch: U and E once per species (2 x 624 B/site) "
                                              "+ 1152 B/site per vector stream",
                         "design_bytes_incl_cached_blocks": {
                             "GB_per_launch": design_bytes / max(1, sten["launches"]) / 1e9,
                             "GBps": design_bytes / (sten["ms"] / 1000.0) / 1e9 if sten["ms"] > 0 else None,
                             "frac": (design_bytes / (sten["ms"] / 1000.0) / 1e9 / peak) if sten["ms"] > 0 else None},
                         "launches": sten["launches"], "avg_launch_ms": sten["ms"] / max(1, sten["launches"]),
                         "step_algorithmic_GBps": step_bytes / (ms_per_step / 1000.0) / 1e9,
                         "byte_model_of_the_plan": model,
                         "fp64": {"flops_per_site_per_launch": flops_site, "achieved_tflops": fp64_achieved,
                                  "peak_tflops": p64, "peak_source": "measured (cuBLAS DGEMM, torch.matmul)",
                                  "frac": fp64_achieved / p64 if fp64_achieved else None}},
            "leapfrog_only": leapfrog_summary(lf_ms, lf_prof, V, peak, p64),
            "kernel_classes": prof,
            "stencil": stencil,
            "cn": {"iterations_per_step": float(np.mean(its)) if its else None,
                   "matvecs_per_step": float(np.mean([s["matvecs"] for s in iters])) if iters else None,
                   "max_rel_residual": max(s["max_rel_residual"] for s in iters) if iters else None,
                   "norms": [norm_q, norm_a]},
            "clocks": clk, "e2e": e2e, "gpu_launches": int(sum(v["launches"] for v in prof.values())),
            "cn_forms_at_1e-10": forms,
            "batching_ensemble": ensemble,
            "precision_drift": drift,
            "thermal_initial_condition": thermal,
            "gluon_distribution": gluon,
        }
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_sample(min(L, 64))
        print(json.dumps(line), flush=True)
    del h, g
    nrqcd.FinalizeModule()
    lattice.FinalizeModule()
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
