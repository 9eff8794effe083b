#!/usr/bin/env python
"""ISF time-step benchmark on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl isf|reference]

Workload: the leapfrogging vortex-ring configuration, 256x128x128 grid on a
10x5x5 torus, hbar 0.1, dt 1/24, 4 194 304 particles seeded in thin tori
around the rings (no nozzle: one pressure projection per step).  A step is one
simloop body (examples/benchmark.jl:46-65 of the reference without the jet
lines): Schroedinger flow, normalize, pressure projection, velocity one-form
+ staggered sharp, RK4 advection of every particle slot.

Printed JSON (rank 0): value = steps/s of the whole job (N independent
replicas for N > 1, "scaling": "weak"), timed with CUDA events on the
library's stream over exactly K steps after W warm-up steps, max over ranks.
The working set (psi 64 MiB, velocity 65 MiB, particles 48 MiB, divergence
16 MiB, half spectrum 18 MiB) is larger than the 126 MB L2, so no flush is
needed between steps.

--impl reference times the CPU restatement of the reference's path (FP32,
OpenMP over all host cores) on the same workload: the reference itself is
Julia 0.6 code that cannot run here.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ISF steps/s (256x128x128, 4M particles) & adjoint/batched vs plain, 1 B200"
UNIT = "steps/s"
WORKLOAD = "vortex_rings_256x128x128_4194304_particles"
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes of each launch site, per grid cell (and per particle slot
# for the advection): every array a kernel must read or write, once.  The
# Poisson passes work on the half spectrum of the real divergence, nx/2+1
# complex64 values per x row (HALF_SPECTRUM bytes per cell; the row padding to
# a multiple of 16 is not counted).
HALF_SPECTRUM = 8.0 * (256 // 2 + 1) / 256
SITE_BYTES_PER_CELL = {
    "schroedinger x fwd": 32, "schroedinger y fwd": 32, "schroedinger z mask": 32, "schroedinger y inv": 32,
    "schroedinger x inv": 32,                      # psi read + write (normalize fused into x inv)
    "projection div": 20,                          # psi read, f write
    "projection x fwd": 4 + HALF_SPECTRUM,         # f read, half spectrum write
    "projection y fwd": 2 * HALF_SPECTRUM, "projection z fac": 2 * HALF_SPECTRUM,
    "projection y inv": 2 * HALF_SPECTRUM,         # half spectrum read + write
    "projection yz planes": 2 * HALF_SPECTRUM,     # k-major half spectrum read + write once
    "projection x inv + gauge": HALF_SPECTRUM + 32,   # half spectrum read, psi read + write
    "step one_form": 28,                           # psi read, velocity write (3 floats)
    "step advect": 12,                             # velocity read (+ 24 B per particle slot)
}
# the whole-step numerator keeps the per-step convention of one read + write
# of each operand per fused pass: 64 (Schroedinger) + 36 (normalize, one-form,
# div) + 32 (Poisson) + 52 (gauge, one-form) + 12 (particle gathers)
STEP_BYTES_PER_CELL = 196      # no-jet step: 64 + 36 + 32 + 52 + 12
STEP_BYTES_PER_PARTICLE = 24   # position read + write


def rank_max(x: float, world: int, device) -> float:
    """The maximum of x over the ranks of the process group (x itself on one
    rank): the job is as slow as its slowest replica."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(steps: int, ms_max: float, world: int) -> float:
    """Steps per second of the whole job: every replica ran `steps` steps
    within ms_max milliseconds (the max over ranks)."""
    return world * steps / (ms_max / 1000.0)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["isf", "reference"], default="isf")
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-ensemble comparison")
    ap.add_argument("--batch-only", action="store_true",
                    help="run only the batched-ensemble comparison and print its JSON object (no contract line)")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint cost measurement")
    ap.add_argument("--no-matlabport", action="store_true", help="skip the MatlabPort front-end loop")
    ap.add_argument("--tma", action="store_true", help="stage the z pass pencils with TMA copies into shared memory")
    ap.add_argument("--order-every", type=int, default=0,
                    help="advect through a cell-sorted slot permutation rebuilt every N steps (0: storage order)")
    return ap.parse_args()


def measured_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_table():
    """dram bytes per launch per site from the committed ncu summary, if any."""
    out = {}
    p = os.path.join(ROOT, "profiles", "ncu_traffic_c3.txt")
    if os.path.exists(p):
        for line in open(p):
            parts = line.strip().split("|")
            if len(parts) >= 4 and parts[1].strip().startswith("site:"):
                try:
                    out[parts[1].strip()[5:].strip()] = float(parts[2])
                except ValueError:
                    pass
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        """Start sampling every 50 ms; returns once the first sample has
        arrived (nvidia-smi takes a while to start), so the samples cover the
        timed region that follows."""
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.idx), "-lms", "50"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.monotonic() + 5.0
            while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t0 = time.monotonic()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def stop(self):
        """Samples taken from start() until one sampling period after the
        timed region (at least the first sample after it)."""
        if not self.proc:
            return None
        t1 = time.monotonic()
        deadline = t1 + 1.0
        while time.monotonic() < deadline and not any(t > t1 for t, _ in self.lines):
            time.sleep(0.01)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.t.join(timeout=2)
        after = [t for t, _ in self.lines if t > t1]
        t_end = max(t1 + 0.06, min(after)) if after else t1 + 0.06
        self.lines = [ln for t, ln in self.lines if self.t0 <= t <= t_end]
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def setup_workload(cfgs):
    c = cfgs.CONFIGS["C3"]
    psi0 = cfgs.vortex_rings_psi(c).astype(np.float32)
    parts = cfgs.torus_particles(c["particles"], c["rings"], c["ring_yz"], c["torus_minor"], c["seed"])
    parts = parts[cfgs.cell_sort_order(parts, c["L"], c["dims"])].astype(np.float32)
    return c, np.ascontiguousarray(psi0), np.ascontiguousarray(parts)


def cpu_baseline(c, psi0, parts0, budget_s, steps_cap=None):
    """FP32 restatement of the reference path on the host cores."""
    import __graft_entry__ as ge
    oracle = ge.load_oracle()
    oracle.build()
    o = oracle.Oracle(c["L"], c["dims"], c["hbar"], c["dt"], prec=32)
    psi = psi0.copy()
    parts = parts0.copy()
    t0 = time.perf_counter()
    o.step(psi, parts, None)
    t1 = time.perf_counter() - t0
    n = max(1, int(budget_s / max(t1, 1e-3)))
    if steps_cap is not None:
        n = min(n, steps_cap)
    t0 = time.perf_counter()
    for _ in range(n):
        o.step(psi, parts, None)
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": UNIT, "cores": oracle.num_threads(), "kind": "port",
            "sample": f"{n} step(s) of {WORKLOAD} after 1 untimed step, FP32 C++ restatement of "
                      f"src/parallel.jl (OpenMP, own FFT; FFTW is absent)"}


def oracle_parity(pkg, c, psi0, parts0, local, steps=10, every=16):
    """The GPU step against the FP64 oracle on the bench workload: `steps`
    steps from the same initial state; psi's relative L2 error and the largest
    particle error (as a fraction of the box) over every `every`-th slot, for
    the particles whose FP64 sample points stayed 1e-4 cells from every face
    (where FP32 and FP64 may pick different cells).  Part of the CPU leg: the
    oracle only checks."""
    import torch
    import __graft_entry__ as ge
    oracle = ge.load_oracle()
    oracle.build()
    orc = oracle.Oracle(c["L"], c["dims"], c["hbar"], c["dt"], prec=64)
    psi64 = psi0.astype(np.float64)
    sub = slice(None, None, every)
    p64 = parts0[sub].astype(np.float64)
    margin = np.full(len(p64), 1e30)
    isf = pkg.ISF(c["L"], c["dims"], c["hbar"], c["dt"], device=local)
    psi = torch.from_numpy(psi0).to(f"cuda:{local}")
    parts = torch.from_numpy(parts0).to(f"cuda:{local}")
    for _ in range(steps):
        pkg.step(isf, psi, parts, None)
        m = np.zeros(len(p64))
        orc.step(psi64, p64, None, margin=m)
        margin = np.minimum(margin, m)
    isf.sync()
    pg = parts.cpu().numpy().astype(np.float64)[sub]
    g = psi.cpu().numpy().astype(np.float64)
    psi_err = float(np.linalg.norm(g - psi64) / np.linalg.norm(psi64))
    both = (pg[:, 0] >= 0) & (p64[:, 0] >= 0)
    ok = both & (margin > 1e-4)
    err = np.abs(pg - p64).max(axis=1) / min(c["L"])
    isf.close()
    bar = 1e-4
    perr = float(err[ok].max()) if ok.any() else None
    mismatch = int(((pg[:, 0] >= 0) != (p64[:, 0] >= 0)).sum())
    # every error against the bar; alive/dead disagreements as a fraction of the sampled slots
    within = {"psi": psi_err <= bar, "particles": perr is not None and perr <= bar,
              "alive": mismatch <= bar * len(p64)}
    res = {"steps": steps, "oracle": "FP64 restatement (oracle/isf_oracle.cpp)", "psi_rel_l2": psi_err,
           "particles_max_err_of_box": perr, "particles_checked": int(ok.sum()), "particles_sampled": int(len(p64)),
           "alive_mismatch": mismatch, "sample": f"every {every}th particle slot", "bar": bar,
           "within_bar": within, "ok": all(within.values())}
    if not res["ok"]:
        print(f"bench: PARITY FAILURE against the FP64 oracle: {json.dumps(res)}", file=sys.stderr, flush=True)
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import __graft_entry__ as ge
    cfgs = importlib.import_module(ge.load_package().__name__ + ".configs")
    c, psi0, parts0 = setup_workload(cfgs)
    budget = max(20.0, min(120.0, 0.5 * (args.steps + args.warmup)))
    cb = cpu_baseline(c, psi0, parts0, budget, steps_cap=args.steps)
    v = cb["value"]
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "grid": list(c["dims"]), "particles": c["particles"],
                       "parallelism": "host cores (OpenMP)"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def batched_vs_plain(pkg, cfgs, steps, warmup, local):
    """The batched ensemble (64 jets on uneven grids, 65 536 particles each,
    one CUDA graph per step) against the same 64 simulations run one after
    another through single-simulation handles (isf_step per step, each run
    synchronised before the next starts).  Both are timed with CUDA events;
    the sequential runs are bracketed on the legacy default stream, which the
    handles' blocking streams are ordered with."""
    import ctypes as C
    import torch
    sims, psi0, parts0 = cfgs.ensemble(nsims=64, seed=3, nslots=65536)
    dev = f"cuda:{local}"
    b = pkg.ISFBatch(sims, device=local, tune=True)
    for i in range(len(sims)):
        b.set_psi(i, torch.from_numpy(psi0[i]).to(dev))
        b.set_particles(i, torch.from_numpy(parts0[i]).to(dev))
    b.init_jet(10)
    b.step(warmup)
    b.sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(b.stream)
    b.step(steps)
    e1.record(b.stream)
    e1.synchronize()
    t_batch = e0.elapsed_time(e1)
    ncls, _ = b.classes()
    tiles = {str(c): b.tiles(c) for c in range(ncls)}
    # the same ensemble as one persistent launch per call (all `steps` steps
    # as work items of one kernel, bounded device-side waits between passes)
    persistent = None
    try:
        b.set_persistent(True)
        b.step(warmup)
        b.sync()
        e0.record(b.stream)
        b.step(steps)
        e1.record(b.stream)
        e1.synchronize()
        b.sync()
        t_pers = e0.elapsed_time(e1)
        persistent = {"value": len(sims) * steps / (t_pers / 1000.0), "unit": "sim-steps/s",
                      "ms_per_ensemble_step": t_pers / steps, "launches_per_call": 1,
                      "what": "isf_batch_set_persistent: one graph-captured launch of the persistent kernel per "
                              "isf_batch_step call"}
    except pkg.ISFError as err:
        persistent = {"unavailable": str(err)}
    b.close()

    # the same simulations, one plain run after another
    runs = []
    for i, s in enumerate(sims):
        h = pkg.ISF(s["physical_size"], s["dims"], s["hbar"], s["dt"], device=local)
        psi = torch.from_numpy(psi0[i]).to(dev)
        parts = torch.from_numpy(parts0[i]).to(dev)
        j = s["jet"]
        for _ in range(10):
            pkg.restrict_velocity(h, psi, j["kvec"], None, 0.0, nozzle=(j["cen"], j["len"], j["rad"]),
                                  phase_mode=j["phase_mode"])
            pkg.pressure_project(h, psi)
        dt32 = np.float32(s["dt"])
        args = []
        for k in range(1, warmup + steps + 1):
            t = np.float32(k) * dt32
            args.append(pkg.step_args(dict(kvec=j["kvec"], omega_t=float(np.float32(j["omega"]) * t), cen=j["cen"],
                                           len=j["len"], rad=j["rad"], phase_mode=j["phase_mode"],
                                           emit_mode=j["emit_mode"], emit_count=0, seed=j["seed"], counter=k)))
        runs.append((h, psi, parts, args))
    for h, psi, parts, args in runs:
        for a in args[:warmup]:
            pkg._lib.check(h.L.isf_step(h.h, C.c_void_p(psi.data_ptr()), C.c_void_p(parts.data_ptr()),
                                        parts.shape[0], C.byref(a)), h.h)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for h, psi, parts, args in runs:
        pp, qq, n = C.c_void_p(psi.data_ptr()), C.c_void_p(parts.data_ptr()), parts.shape[0]
        for a in args[warmup:]:
            h.L.isf_step(h.h, pp, qq, n, C.byref(a))
        pkg._lib.check(h.L.isf_sync(h.h), h.h)
    f1.record()
    f1.synchronize()
    t_seq = f0.elapsed_time(f1)
    for h, *_ in runs:
        h.close()
    n = len(sims)
    return {"workload": "ensemble_64_jets_32^3-96x48x48_65536_particles", "sims": n, "steps": steps,
            "grids": {str(g): sum(1 for s in sims if tuple(s["dims"]) == g[0]) for g in cfgs.ENSEMBLE_GRIDS},
            "value": n * steps / (t_batch / 1000.0), "unit": "sim-steps/s",
            "sequential_value": n * steps / (t_seq / 1000.0), "ratio_vs_sequential": t_seq / t_batch,
            "ms_per_ensemble_step": t_batch / steps, "classes": ncls, "tiles": tiles,
            "persistent": (dict(persistent, ratio_vs_sequential=t_seq / (n * steps / persistent["value"] * 1000.0))
                           if persistent and "value" in persistent else persistent)}


def sharded_ensemble(pkg, cfgs, steps, warmup, rank, world, local):
    """The C4 ensemble spread over the ranks: each rank steps its share of the
    64 jets (configs.shard, balanced by bytes per step) as one batch on its own
    GPU, with no collective on the data path.  Timed with CUDA events on each
    batch's stream; the whole job's rate uses the slowest rank."""
    import torch
    sims, psi0, parts0 = cfgs.ensemble(nsims=64, seed=3, nslots=65536)
    mine = cfgs.shard([cfgs.sim_cost(s) for s in sims], world)[rank]
    dev = f"cuda:{local}"
    b = pkg.ISFBatch([sims[i] for i in mine], device=local, tune=True)
    for k, i in enumerate(mine):
        b.set_psi(k, torch.from_numpy(psi0[i]).to(dev))
        b.set_particles(k, torch.from_numpy(parts0[i]).to(dev))
    b.init_jet(10)
    b.step(warmup)
    b.sync()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(b.stream)
    b.step(steps)
    e1.record(b.stream)
    e1.synchronize()
    ms = rank_max(e0.elapsed_time(e1), world, dev)
    b.close()
    return {"workload": "ensemble_64_jets_32^3-96x48x48_65536_particles", "sims": len(sims), "ranks": world,
            "sims_this_rank": len(mine), "steps": steps, "sim_steps_per_s": len(sims) * steps / (ms / 1000.0),
            "what": "the 64 simulations split over the ranks by bytes per step, one batch per GPU, "
                    "max over ranks"}


MATLAB_CFG = dict(L=(4, 2, 2), dims=(64, 32, 32), hbar=0.1, dt=1 / 48, slots=20000, births=10)


def matlabport_loop(pkg, cfgs, steps, warmup, local):
    """The MatlabPort driver loop (examples/matlabport/simple.jl:20-124) on the
    64x32x32 jet through the FP64 structure-of-arrays front-end: FP64 psi1,
    psi2 and velocity arrays between the calls, 20 000 particle slots, 10
    births per step, removethedead! every step.  Device-timed with CUDA events
    on the legacy default stream, which the library's blocking streams are
    ordered with."""
    import torch
    mp = pkg.matlabport
    c = MATLAB_CFG
    L, dims, hbar, dt = c["L"], c["dims"], c["hbar"], c["dt"]
    noz = cfgs.JET_NOZZLE
    vjet = np.array([1.0, 0.0, 0.0])
    kvec, omega = vjet / hbar, float(np.sum(vjet ** 2) / (2 * hbar))
    obj = mp.ISF(L, dims, hbar, dt, device=local)
    isjet = mp.is_jet(obj, noz["cen"], noz["len"], noz["rad"])
    dev = f"cuda:{local}"
    a1, a2 = mp.Normalize(torch.ones(dims, dtype=torch.complex128, device=dev),
                          0.01 * torch.ones(dims, dtype=torch.complex128, device=dev))
    for _ in range(10):
        a1, a2 = mp.restrict(obj, a1, a2, isjet, kvec, 0.0)
        a1, a2 = mp.PressureProject(obj, a1, a2)
    slots, nb = c["slots"], c["births"]
    p = mp.Particles(np.zeros(slots), np.zeros(slots), np.zeros(slots), device=local)

    def body(it, a1, a2):
        t = it * dt
        a1, a2 = mp.SchroedingerFlow(obj, a1, a2)
        a1, a2 = mp.Normalize(a1, a2)
        a1, a2 = mp.PressureProject(obj, a1, a2)
        a1, a2 = mp.restrict(obj, a1, a2, isjet, kvec, omega * t)
        a1, a2 = mp.PressureProject(obj, a1, a2)
        mp.add_ring(p, nb, noz["cen"], noz["rad"], seed=0, counter=it)
        mp.remove_dead(p, obj)
        vx, vy, vz = mp.VelocityOneForm(obj, a1, a2, obj.hbar)
        vx, vy, vz = mp.StaggeredSharp(obj, vx, vy, vz)
        mp.StaggeredAdvect(p, obj, vx, vy, vz, obj.dt)
        return a1, a2

    steps = min(steps, (slots - 1) // nb - warmup - 1)
    for it in range(1, warmup + 1):
        a1, a2 = body(it, a1, a2)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for it in range(warmup + 1, warmup + steps + 1):
        a1, a2 = body(it, a1, a2)
    e1.record()
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"workload": "matlabport_driver_jet_64x32x32_20000_slots_10_births_per_step", "steps": steps,
            "steps_per_s": 1000.0 / ms, "ms_per_step": ms, "live_particles": int(p.active.numel()),
            "what": "SchroedingerFlow, Normalize, PressureProject, restrict, PressureProject, add_ring, "
                    "remove_dead (one host read of the live count), VelocityOneForm, StaggeredSharp, "
                    "StaggeredAdvect on FP64 arrays"}


def matlabport_cpu_baseline(cfgs, k=3):
    """The same driver loop in the FP64 numpy restatement of MatlabPort.jl
    (oracle/matlabport.py) on the host, k steps: steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import matlabport as orc_mp
    c = MATLAB_CFG
    noz = cfgs.JET_NOZZLE
    vjet = np.array([1.0, 0.0, 0.0])
    kvec, omega = vjet / c["hbar"], float(np.sum(vjet ** 2) / (2 * c["hbar"]))
    oo = orc_mp.MatlabISF(c["L"], c["dims"], c["hbar"], c["dt"])
    isjet = orc_mp.is_jet(oo, noz["cen"], noz["len"], noz["rad"])
    b1, b2 = orc_mp.normalize(np.ones(c["dims"], np.complex128), 0.01 * np.ones(c["dims"], np.complex128))
    x, y, z = (np.zeros(c["slots"], np.float32) for _ in range(3))
    n, act = 0, np.zeros(0, np.int64)
    rng = np.random.default_rng(0)
    t0 = time.perf_counter()
    for it in range(1, k + 1):
        th = rng.uniform(0, 2 * np.pi, c["births"]).astype(np.float32)
        births = (np.full(c["births"], noz["cen"][0], np.float32),
                  (noz["cen"][1] + 0.9 * noz["rad"] * np.cos(th)).astype(np.float32),
                  (noz["cen"][2] + 0.9 * noz["rad"] * np.sin(th)).astype(np.float32))
        b1, b2, n, act = orc_mp.driver_step(oo, b1, b2, isjet, kvec, omega * it * c["dt"], x, y, z, n, act, births)
    return {"value": k / (time.perf_counter() - t0), "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": f"{k} steps of the same loop in numpy FP64"}


def adjoint_vs_forward(pkg, cfgs, reps, local):
    """The particle-loss gradient of the 64x32x32 jet (65 536 particles
    uniform in the box, 10 initialisation projections, 50 steps, psi
    checkpointed every 10 steps; isf_adj_gradient) against the forward alone
    (isf_adj_loss, the same 50 steps).  CUDA events on the handle's stream."""
    import torch
    c = cfgs.CONFIGS["C1"]
    isf = pkg.ISF(c["L"], c["dims"], c["hbar"], c["dt"], device=local)
    dev = f"cuda:{local}"
    kvec, omega = cfgs.jet_omega(c["hbar"])
    noz = cfgs.JET_NOZZLE
    prob = pkg.adj_problem(50, 10, kvec, omega, (noz["cen"], noz["len"], noz["rad"]), init_iters=10)
    rng = np.random.Generator(np.random.Philox(4))
    P = 65536
    p0 = torch.tensor(rng.uniform(0, 1, (P, 3)) * np.asarray(c["L"]), dtype=torch.float32, device=dev)
    psi0 = torch.from_numpy(cfgs.jet_init_psi(c["dims"]).astype(np.float32)).to(dev)
    tgt = p0 + torch.tensor(rng.normal(0, 0.1, (P, 3)), dtype=torch.float32, device=dev)
    pkg.adj_gradient(isf, prob, psi0, p0, tgt)   # warm-up (allocates the tape)
    pkg.adj_loss(isf, prob, psi0, p0, tgt)
    isf.sync()
    s = isf.stream

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(reps):
            fn()
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / reps

    t_fwd = timed(lambda: pkg.adj_loss(isf, prob, psi0, p0, tgt))
    t_grad = timed(lambda: pkg.adj_gradient(isf, prob, psi0, p0, tgt))
    isf.close()
    return {"workload": "jet_64x32x32_65536_particles_50_steps_checkpoint_10", "forward_ms": t_fwd,
            "gradient_ms": t_grad, "ratio_gradient_vs_forward": t_grad / t_fwd,
            "what": "isf_adj_gradient (forward with checkpoints + segment recompute + reverse) / isf_adj_loss"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    import __graft_entry__ as ge

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    pkg = ge.load_package()
    cfgs = importlib.import_module(pkg.__name__ + ".configs")
    if args.batch_only:
        print(json.dumps(batched_vs_plain(pkg, cfgs, min(args.steps, 100), args.warmup, local)), flush=True)
        return
    c, psi0, parts0 = setup_workload(cfgs)
    P = parts0.shape[0]
    ncells = int(np.prod(c["dims"]))

    isf = pkg.ISF(c["L"], c["dims"], c["hbar"], c["dt"], device=local, flags=pkg.FLAG_TMA_Z_PASS if args.tma else 0)
    isf.set_particle_order(args.order_every)
    s = isf.stream
    psi = torch.from_numpy(psi0).to(f"cuda:{local}")
    parts = torch.from_numpy(parts0).to(f"cuda:{local}")
    torch.cuda.synchronize()

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        return rank_max(x, world, f"cuda:{local}")

    # ---- device-resident timing
    for _ in range(args.warmup):
        pkg.step(isf, psi, parts, None)
    isf.sync()
    barrier()
    torch.cuda.synchronize()
    launches0 = isf.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = ev(), ev()
    e0.record(s)
    for _ in range(args.steps):
        pkg.step(isf, psi, parts, None)
    isf.join()  # the last step's advection, queued on the particle stream
    e1.record(s)
    e1.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    gpu_launches = isf.launch_count() - launches0
    ms = max_over_ranks(ms)
    value = whole_job_rate(args.steps, ms, world)
    ms_per_step = ms / args.steps

    # ---- per-launch-site timing over a second pass of the same window
    # (state reset to the initial condition, same warm-up) for the roofline
    psi.copy_(torch.from_numpy(psi0))
    parts.copy_(torch.from_numpy(parts0))
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        pkg.step(isf, psi, parts, None)
    isf.sync()
    isf.profile_start()
    for _ in range(args.steps):
        pkg.step(isf, psi, parts, None)
        # each launch timed alone: the advection on the particle stream is
        # joined before the next step's passes are queued
        isf.join()
    sites = isf.profile_stop()
    total_site_ms = sum(v[0] for v in sites.values())
    dom = max(sites, key=lambda k: sites[k][0])
    dom_ms, dom_n = sites[dom]
    dom_bytes = SITE_BYTES_PER_CELL.get(dom, 0) * ncells + (STEP_BYTES_PER_PARTICLE * P if dom == "step advect" else 0)
    peak, peak_kind = measured_hbm()
    achieved = dom_bytes / (dom_ms / dom_n / 1000.0) / 1e9
    traffic = traffic_table().get(dom)
    step_bytes = STEP_BYTES_PER_CELL * ncells + STEP_BYTES_PER_PARTICLE * P
    step_achieved = step_bytes / (ms_per_step / 1000.0) / 1e9

    # ---- end to end through the C ABI with host buffers
    e2e = None
    if not args.no_e2e:
        h_psi = torch.from_numpy(psi0).pin_memory()
        h_parts = torch.from_numpy(parts0).pin_memory()
        o_psi = torch.empty_like(h_psi).pin_memory()
        o_parts = torch.empty_like(h_parts).pin_memory()
        import ctypes as C
        L = isf.L
        barrier()
        torch.cuda.synchronize()
        f0, f1 = ev(), ev()
        f0.record(s)
        pkg._lib.check(L.isf_memcpy_h2d(isf.h, C.c_void_p(psi.data_ptr()), C.c_void_p(h_psi.data_ptr()),
                                        h_psi.numel() * 4), isf.h)
        pkg._lib.check(L.isf_memcpy_h2d(isf.h, C.c_void_p(parts.data_ptr()), C.c_void_p(h_parts.data_ptr()),
                                        h_parts.numel() * 4), isf.h)
        # every step's result (clamp events, live particles: 16 bytes) is read
        # back into pinned host memory, queued behind the step
        res = torch.zeros((args.steps, 2), dtype=torch.int64).pin_memory()
        for k in range(args.steps):
            pkg.step(isf, psi, parts, None)
            isf.counters_async(res[k], reset=True)
        pkg._lib.check(L.isf_memcpy_d2h(isf.h, C.c_void_p(o_psi.data_ptr()), C.c_void_p(psi.data_ptr()),
                                        o_psi.numel() * 4), isf.h)
        pkg._lib.check(L.isf_memcpy_d2h(isf.h, C.c_void_p(o_parts.data_ptr()), C.c_void_p(parts.data_ptr()),
                                        o_parts.numel() * 4), isf.h)
        f1.record(s)
        f1.synchronize()
        live = int(res[-1, 1])
        ems = max_over_ranks(f0.elapsed_time(f1))
        state = (h_psi.numel() + h_parts.numel()) * 4
        e2e = {"value": whole_job_rate(args.steps, ems, world), "unit": UNIT,
               "h2d_bytes_per_step": state / args.steps, "d2h_bytes_per_step": 16 + state / args.steps,
               "what": "isf_memcpy_h2d of psi0 + particles, K x (isf_step + 16-byte counter read into pinned "
                       "host memory, isf_counters_async), isf_memcpy_d2h of psi + particles",
               "live_particles_last_step": live}
    sharded = None
    if world > 1 and not args.no_batch:
        sharded = sharded_ensemble(pkg, cfgs, min(args.steps, 100), args.warmup, rank, world, local)
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    del isf
    batched = None
    if not args.no_batch:
        batched = batched_vs_plain(pkg, cfgs, min(args.steps, 100), args.warmup, local)
    adjoint = None
    if not args.no_adjoint:
        adjoint = adjoint_vs_forward(pkg, cfgs, 3, local)
    matlab = None
    if not args.no_matlabport:
        matlab = matlabport_loop(pkg, cfgs, min(args.steps, 200), args.warmup, local)

    cb = None
    parity = None
    if not args.no_cpu:
        cb = cpu_baseline(c, psi0, parts0, args.cpu_seconds)
        parity = oracle_parity(pkg, c, psi0, parts0, local)
        if matlab is not None:
            matlab["cpu_baseline"] = matlabport_cpu_baseline(cfgs)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "grid": list(c["dims"]), "torus": list(c["L"]), "hbar": c["hbar"],
                   "dt": c["dt"], "particles": P, "jet": False, "particle_order_every": args.order_every, "tma_z_pass": args.tma,
                   "l2": "inputs larger than L2: psi 64 MiB + velocity 65 MiB + particles 48 MiB + f 16 MiB + half spectrum 18 MiB",
                   "parallelism": "replicas" if world > 1 else "single"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                     "launch_ms": dom_ms / dom_n, "share_of_step": dom_ms / total_site_ms},
        "step_roofline": {"algorithmic_bytes_per_step": step_bytes, "achieved": step_achieved, "peak": peak,
                          "unit": "GB/s", "frac": step_achieved / peak},
        "kernels_ms_per_step": {k: v[0] / args.steps for k, v in sorted(sites.items(), key=lambda kv: -kv[1][0])},
        "e2e": e2e, "gpu_launches": gpu_launches, "clocks": clk, "cpu_baseline": cb,
        "batched": batched, "batched_sharded": sharded, "adjoint": adjoint, "matlabport": matlab, "parity": parity,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
