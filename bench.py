#!/usr/bin/env python
"""Benchmark of the SELM step: fluid-cell-steps/s at 128^3 with 1e5 monomers.

Workload (the large single-instance configuration): 1000 FENE chains x 100
monomers (K=30, R0=1.5, WCA sigma=eps=1) seeded as random walks in a periodic
box L=128 on a 128^3 grid, kT=1, dt=0.005, mu=rho=1, synthetic (seeded)
positions.  A "step" is one full SELM step: monomer binning, interpolation +
monomer update, spreading, the fluid update (FFT, projection, viscous step,
thermal noise), and the device conservative forces.

``value`` is the FP32 fused form, whole job (all ranks), device-timed with
CUDA events around each step (L2 flushed before every timed step, outside the
events), max over ranks.  The plain FP64 form (reference structure) and the
FP64 fused form are timed on the same workload beside it.  ``e2e`` is the
same metric through the public API with host buffers: set the monomer state
from pinned host memory, step, read the monomer state back, every step.

``--impl reference`` times the reference's CPU step (the reference's own
source built against single-rank shims when available, else the FP64 port in
oracle/) on all the host's hardware threads: one single-rank instance of the
same workload per thread, run concurrently, their cell-steps summed over the
common window (torchrun rank 0 only).
"""
from __future__ import annotations

import argparse
from dataclasses import replace
import json
import os
import statistics
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

HBM_FALLBACK_GBS = 6650.0
_T0 = time.time()


def log(msg: str) -> None:
    print(f"[bench {time.time() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


# --------------------------------------------------------------------------- clocks
class Clocks:
    """SM clock and clock-event-reason sampler for the timed region.

    Polls NVML from a background thread every few milliseconds, so that a
    timed region of a few tens of milliseconds still gets samples; reports no
    samples (and why) when NVML cannot be used."""

    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}

    def __init__(self, device_index: int, period_s: float = 0.002):
        self.device_index = device_index
        self.period = period_s
        self.samples = []
        self.smax = None
        self.stop_flag = None
        self.thread = None
        self.error = None

    def _handle(self, nv):
        import torch
        try:
            pr = torch.cuda.get_device_properties(self.device_index)
            bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
            return nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv.nvmlDeviceGetHandleByIndex(self.device_index)

    def start(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception as e:  # no NVML: no samples
            self.error = f"nvml unavailable: {type(e).__name__}"
            return
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
        self.stop_flag = threading.Event()

        def run():
            while True:
                try:
                    self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(get_reasons(h))))
                except Exception as e:
                    self.error = f"nvml query failed: {type(e).__name__}"
                    return
                if self.stop_flag.wait(self.period):
                    return

        self.thread = threading.Thread(target=run, daemon=True)
        self.thread.start()
        while not self.samples and self.thread.is_alive():  # at least one sample before the region starts
            time.sleep(self.period)

    def stop(self):
        if self.thread is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "note": self.error}
        self.stop_flag.set()
        self.thread.join(timeout=5)
        sm = [c for c, _ in self.samples]
        reasons = sorted({n for _, r in self.samples for n, b in self.REASONS.items() if r & b})
        out = {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax, "reasons": reasons,
               "samples": len(sm), "source": "nvml"}
        if self.error:
            out["note"] = self.error
        return out


# --------------------------------------------------------------------------- helpers
def algorithmic_bytes(kernel: str, N: int, N2: int, M: int, s: int, U: int) -> float:
    """Compulsory DRAM bytes of one launch (one job)."""
    c = 2 * s
    table = {
        "xy_forward": 3 * N * s + 3 * N2 * c,
        "z_update": 4 * 3 * N2 * c,
        "xy_inverse": 3 * N2 * c + 3 * N * s,
        "spread": 3 * N * s + M * (24 + 24 + 4),
        "interp_update": 3 * U * s + M * (24 + 24 + 48 + 48 + 8 + 24 + 4),
        "forces": M * (24 + 24),
        "bin": M * (24 + 4 * 5),
    }
    return float(table.get(kernel, 0.0))


def stencil_union(x: np.ndarray, n: int, lo: float, dx: float) -> int:
    """Distinct grid points read by the interpolation (union of staggered 4^3 stencils)."""
    g = (x - lo) / dx
    pts = set()
    keys = []
    for d in range(3):
        sh = np.where(np.arange(3) == d, 0.0, 0.5)
        base = np.floor(g - sh).astype(np.int64) - 1
        off = np.arange(4)
        ix = (base[:, 0, None, None, None] + off[None, :, None, None]) % n
        iy = (base[:, 1, None, None, None] + off[None, None, :, None]) % n
        iz = (base[:, 2, None, None, None] + off[None, None, None, :]) % n
        keys.append(((d * n + iz) * n + iy) * n + ix)
    del pts
    return int(np.unique(np.concatenate([k.ravel() for k in keys])).size)


def traffic_from_profiles(kernel: str, form: str, N: int):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    e = d.get(form, {}).get(kernel)
    if not e:
        return None
    return float(e["bytes_per_launch"]) * (N / float(e["cells"]))


# --------------------------------------------------------------------------- our arm
def headline_config(n, M, world):
    """The workload the headline line is quoted on; both arms print this same dict."""
    return {"workload": "large single instance: 1000 FENE chains x 100 monomers, L=128, 128^3 grid, "
                        "kT=1, dt=0.005", "grid": n, "monomers": M, "parallelism": f"replicas x{world}",
            "l2": "GPU arm: flushed (256 MB write) before every timed step; CPU arm: no flush"}


def run_ours(args, rank, world, local_rank):
    import torch

    from monomers2026_b200 import _lib
    from monomers2026_b200 import workloads as W
    from monomers2026_b200.selm import Selm

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    lib = _lib.load()
    log("generating the workload")
    wl = W.config(3, form=args.form, seed=1003 + rank)
    log(f"workload ready: {len(wl.mass)} monomers")
    p = wl.params
    p.SELM_Seed = 1003 + rank
    n = p.numMeshPtsPerDir[0]
    N = n ** 3
    N2 = (n // 2 + 1) * n * n
    M = len(wl.mass)
    # a dedicated stream: the library runs on it and the CUDA events are recorded on it
    # (the handle of torch's default stream is 0, which the library reads as "own stream")
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    def make(form, integrator="inertial"):
        wl.params.form = form
        wl.params.integrator = integrator
        sim = Selm(wl.params, wl.x, wl.mass, topology=wl.topology)
        sim.set_stream(stream.cuda_stream)
        sim.initial()
        return sim

    def timed(sim, K, Wm):
        for _ in range(Wm):
            flush.zero_()
            sim.run(1)
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
        l0 = lib.selm_kernel_launches()
        for k in range(K):
            flush.zero_()
            ev[k][0].record(stream)
            sim.run(1)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
        launches = lib.selm_kernel_launches() - l0
        if world > 1:
            torch.distributed.barrier()
        per = [a.elapsed_time(b) for a, b in ev]
        return per, launches

    def reduce_max(v):
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # ---- autotuner: FFT split and z-kernel occupancy for this shape (a throwaway copy)
    tuned = None
    if args.form != "plain64" and not args.no_autotune:
        from monomers2026_b200.autotune import tune
        wl.params.form = args.form
        tuned = tune(wl)
        log(f"autotune: {tuned['choice']}")

    # ---- headline form, timed with clocks sampled
    sim = make(args.form)
    log("timed steps")
    clk = Clocks(local_rank)
    clk.start()
    per, launches = timed(sim, args.steps, args.warmup)
    clocks = clk.stop()
    total_ms = reduce_max(sum(per))
    value = world * N * args.steps / (total_ms / 1e3)
    status = sim.status()

    log(f"timed: {sum(per) / len(per):.3f} ms/step, status 0x{status:x}")
    # ---- per-kernel times (a separate pass with CUDA events around every kernel)
    sim.profile(True)
    pk = max(5, min(args.steps, 20))
    for _ in range(pk):
        flush.zero_()
        sim.run(1)
    kern = {}
    for name in ("bin", "interp_update", "spread", "xy_forward", "z_update", "xy_inverse", "forces"):
        ms, cnt = sim.profile_read(name)
        if cnt:
            kern[name] = (ms / cnt, cnt // pk)
    sim.profile(False)

    log(f"kernel times: {kern}")
    # ---- end-to-end through the public API with host buffers
    x, v, f = sim.particles()
    xp = torch.empty((M, 3), dtype=torch.float64).pin_memory().numpy()
    vp = torch.empty((M, 3), dtype=torch.float64).pin_memory().numpy()
    fp = torch.empty((M, 3), dtype=torch.float64).pin_memory().numpy()
    mp = torch.empty((M,), dtype=torch.float64).pin_memory().numpy()
    xp[:] = x
    vp[:] = v
    mp[:] = wl.mass
    import ctypes as C

    dp = C.POINTER(C.c_double)
    h = sim._h
    ke = max(5, args.steps // 2)
    for _ in range(2):
        _lib.check(lib.selm_set_particles(h, M, xp.ctypes.data_as(dp), vp.ctypes.data_as(dp), mp.ctypes.data_as(dp)))
        _lib.check(lib.selm_step(h, 1))
        _lib.check(lib.selm_get_particles(h, xp.ctypes.data_as(dp), vp.ctypes.data_as(dp), fp.ctypes.data_as(dp)))
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(ke):
        _lib.check(lib.selm_set_particles(h, M, xp.ctypes.data_as(dp), vp.ctypes.data_as(dp), None))  # masses kept
        _lib.check(lib.selm_step(h, 1))
        _lib.check(lib.selm_get_particles(h, xp.ctypes.data_as(dp), vp.ctypes.data_as(dp), fp.ctypes.data_as(dp)))
    torch.cuda.synchronize()
    e2e_s = reduce_max(time.perf_counter() - t0)
    e2e = {"value": world * N * ke / e2e_s, "unit": "fluid-cell-steps/s", "h2d_bytes_per_step": M * (24 + 24),
           "d2h_bytes_per_step": M * 72, "steps": ke}
    log(f"e2e: {e2e['value']:.3e} cell-steps/s")
    U = stencil_union(xp, n, p.box_lo, (p.box_hi - p.box_lo) / n)
    extras = outputs_and_analysis(sim, lib, stream, p.dt)
    log(f"analysis and output: {extras}")
    sim.final()
    del sim

    # ---- the other forms on the same workload
    forms = {}
    if not args.no_forms:
        for form in ("plain64", "fused64"):
            if form == args.form:
                continue
            s2 = make(form)
            k2 = max(5, args.steps // 2)
            per2, _ = timed(s2, k2, max(3, args.warmup // 2))
            forms[form] = world * N * k2 / (reduce_max(sum(per2)) / 1e3)
            log(f"form {form}: {sum(per2) / k2:.3f} ms/step")
            s2.final()
        # the overdamped (quasi-steady) integrator on the same workload and form
        s2 = make(args.form, "quasi_steady")
        k2 = max(5, args.steps // 2)
        per2, _ = timed(s2, k2, max(3, args.warmup // 2))
        forms[f"{args.form}_quasi_steady"] = world * N * k2 / (reduce_max(sum(per2)) / 1e3)
        log(f"form {args.form} quasi-steady: {sum(per2) / k2:.3f} ms/step")
        s2.final()
        wl.params.integrator = "inertial"
    forms[args.form] = value

    # ---- roofline of the dominant kernel
    s = 4 if args.form == "fused32" else 8
    hbm, peak_kind = peaks()
    dom = max(kern, key=lambda k: kern[k][0] * max(1, kern[k][1])) if kern else None
    roof = None
    if dom:
        ab = algorithmic_bytes(dom, N, N2, M, s, U)
        ach = ab / (kern[dom][0] / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(ach / hbm, 4), "peak_kind": peak_kind, "algorithmic_bytes": ab,
                "traffic": traffic_from_profiles(dom, args.form, N)}
        # the whole step beside it: fluid 30 N s (one compulsory sweep of each field) plus the
        # monomers M (48 + 6 s + 8), over the timed step
        step_bytes = 30.0 * N * s + M * (48 + 6 * s + 8)
        step_ach = step_bytes / (total_ms / args.steps / 1e3) / 1e9
        roof["step"] = {"algorithmic_bytes": step_bytes, "achieved": round(step_ach, 1),
                        "frac": round(step_ach / hbm, 4)}

    # ---- batched ensemble and serving (rank 0 at N=1)
    batched = serving = None
    if rank == 0 and world == 1 and not args.no_batched:
        batched, serving = batched_and_serving(args)
    decomposed = None
    if rank == 0 and world == 1 and not args.no_batched:
        log("decomposed instance (2 slabs, loopback)")
        decomposed = decomposed_check(wl)
        log(f"decomposed: {decomposed}")

    # ---- CPU baseline (rank 0 at N=1): the reference's CPU code on every host thread, a bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        log("CPU baseline")
        cpu = cpu_baseline(wl, budget_s=args.cpu_seconds)
    acc = None
    if rank == 0 and world == 1 and args.form == "fused32" and not args.no_forms:
        log("FP32 against FP64 velocities")
        acc = fp32_accuracy(wl, stream)
        log(f"FP32 error: {acc}")
    ref_gpu = xcheck = None
    if rank == 0 and world == 1 and not args.no_cpu:
        log("reference GPU step and cuFFT cross-check")
        ref_gpu, xcheck = reference_gpu_baseline(wl, kern)
        log(f"reference GPU: {ref_gpu and ref_gpu['ms_per_step']} ms/step; cuFFT: {xcheck}")

    if rank == 0:
        out = {
            "metric": "fluid-cell-steps/s @128^3, 1e5 monomers (FP32 fused form; plain FP64 form beside it)",
            "value": value,
            "unit": "fluid-cell-steps/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32" if args.form == "fused32" else "f64",
            "data": "synthetic (seeded random-walk FENE chains)",
            "config": headline_config(n, M, world),
            "form": args.form,
            "latency_ms": {"p50": float(np.percentile(per, 50)), "p99": float(np.percentile(per, 99))},
            "forms": forms,
            "fp32_vs_plain64": (forms[args.form] / forms["plain64"]) if "plain64" in forms else None,
            "kernels_ms": {k: round(v[0], 5) for k, v in kern.items()},
            "interp_union_points": U,
            "roofline": roof,
            "cpu_baseline": cpu,
            "fp32_vs_fp64_velocity_rel_err": acc,
            "reference_gpu": ref_gpu,
            "cufft_xcheck": xcheck,
            "e2e": e2e,
            "analysis_and_output": extras,
            "autotune": tuned,
            "batched": batched,
            "serving": serving,
            "decomposed": decomposed,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "status_word": status,
        }
        print(json.dumps(out))


def batched_and_serving(args):
    """Batched ensemble (256 replicas over {32,48,64,96}^3, one graph launch per
    step) against the same replicas stepped one after another in the plain FP64
    form; FP32 against FP64 velocities on 8 sampled replicas; a bounded serving
    run at configuration 5 (64 jobs, Poisson arrivals at 200/s, 500-5000
    steps each, HBM budget 150 GB) beside the same jobs run sequentially in
    the plain FP64 form."""
    from monomers2026_b200 import serving as SV
    from monomers2026_b200 import workloads as W
    from monomers2026_b200.selm import Selm

    log("batched ensemble: 256 replicas")
    ens = W.ensemble(256)
    tuned = None
    if not args.no_autotune:
        from monomers2026_b200.autotune import tune_ensemble
        tuned = tune_ensemble(ens)
        log("autotune: " + ", ".join(f"{t['grid']}^3 {t['choice']}" for t in tuned))
    b = SV.run_ensemble(ens, steps=args.batch_steps, warmup=3)
    b["autotune"] = tuned
    log(f"batched: {b['replica_steps_per_s']:.0f} replica-steps/s, step p50 {b['step_ms']['p50']:.2f} ms")
    seq = SV.run_sequential(ens, steps=2, form="plain64")
    b["sequential_plain64_replica_steps_per_s"] = seq["replica_steps_per_s"]
    b["speedup_vs_sequential_plain64"] = b["replica_steps_per_s"] / seq["replica_steps_per_s"]
    log(f"sequential plain64: {seq['replica_steps_per_s']:.0f} replica-steps/s")
    errs = []
    for w in ens[::32][:8]:
        v = {}
        for form in ("fused32", "fused64"):
            s = Selm(replace(w.params, form=form), w.x, w.mass, topology=w.topology)
            s.initial()
            s.run(10)
            v[form] = s.particles()[1]
            s.final()
        errs.append(float(np.abs(v["fused32"] - v["fused64"]).max() / np.abs(v["fused64"]).max()))
    b["fp32_vs_fp64_velocity_rel_err"] = {"max": max(errs), "replicas": len(errs), "steps": 10}
    b["config"] = {"workload": "256 replicas, grid uniform over {32,48,64,96}^3 (L=N), monomers log-uniform "
                               "in 50-2000 as FENE+WCA chains of 50, kT uniform in [0.5,2], own Philox seed each",
                   "form": "fused32", "l2": "not flushed: the ensemble's fields (GBs) exceed L2"}
    log("serving run")
    jobs = SV.serving_jobs(64)
    srv = SV.Server(budget_bytes=150 * 10**9)
    sv = srv.run(jobs)
    srv.final()
    sv["wall_over_device"] = sv["replica_steps_per_s_wall"] / sv["replica_steps_per_s_device"]
    sv["step_p99_over_p50"] = sv["step_ms"]["p99"] / sv["step_ms"]["p50"]
    seq = SV.run_sequential_jobs(jobs, form="plain64")
    sv["sequential_plain64_replica_steps_per_s"] = seq["replica_steps_per_s"]
    sv["speedup_wall_vs_sequential_plain64"] = sv["replica_steps_per_s_wall"] / seq["replica_steps_per_s"]
    sv["config"] = {"workload": "64 jobs, Poisson arrivals at 200/s, grid {32,48,64,96,128}^3 w.p. "
                                ".3/.3/.2/.15/.05, one chain of U[20,5000] monomers, U[500,5000] steps",
                    "budget_bytes": 150 * 10**9, "form": "fused32",
                    "sequential": "the same jobs one after another in plain64, each job's step device-timed "
                                  "over 10 steps and counted for all of its steps"}
    log(f"serving: {sv['jobs']} jobs, wall/device {sv['wall_over_device']:.2f}, "
        f"step p50 {sv['step_ms']['p50']:.2f} p99 {sv['step_ms']['p99']:.2f} ms, "
        f"sequential plain64 {seq['replica_steps_per_s']:.0f} replica-steps/s")
    return b, sv


def decomposed_check(wl, nranks=2, steps=5):
    """The headline workload as one instance over `nranks` z slabs, all in this
    process (loopback transport: the slabs run one after another, so the
    time is an emulation, not a decomposed speed), against the whole
    instance: the largest relative deviation of the monomer and fluid
    velocities after `steps` steps (the interpolation is summed slab by slab;
    everything else is the same kernels on the slabs' parts)."""
    import torch

    from monomers2026_b200.decomposed import Decomposed, LoopbackTransport
    from monomers2026_b200.selm import Selm

    whole = Selm(wl.params, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    whole.initial()
    whole.run(steps)
    _, vw, _ = whole.particles()
    uw = whole.get_field(0)
    whole.final()
    dec = Decomposed(wl.params, wl.x, wl.mass, v=wl.v, topology=wl.topology, transport=LoopbackTransport(nranks))
    dec.initial()
    dec.step(1)  # untimed: first use of the exchange buffers
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dec.step(steps - 1)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / (steps - 1) * 1e3
    _, vd, _ = dec.particles()
    ud = np.concatenate([a for _, a in sorted(dec.velocity().items())], axis=1)
    status = dec.status()
    dec.final()

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))

    return {"slabs": nranks, "steps": steps, "loopback_ms_per_step": round(ms, 3),
            "v_rel_dev": rel(vd, vw), "u_rel_dev": rel(ud, uw), "status": status,
            "note": "slabs stepped one after another in one process; the exchanges are device copies"}


def outputs_and_analysis(sim, lib, stream, dt, samples=20, frames=10):
    """Cost of the on-device analysis (one sample: MSD over 40 lags, S(q) at
    the 16 shortest wavevectors, K_d) on the device, and of writing DCD frames
    (read-back plus file write), on the headline simulation."""
    import ctypes as C
    import tempfile

    import torch

    from monomers2026_b200 import _lib
    from monomers2026_b200.analysis import Analysis, wavevectors
    q = wavevectors(2)[:16]
    an = Analysis(sim, nlag=40, lag_stride=1, qvec=q)
    for _ in range(3):
        an.sample()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(samples):
        an.sample()
    b.record(stream)
    b.synchronize()
    sample_us = 1000.0 * a.elapsed_time(b) / samples
    an.close()
    with tempfile.TemporaryDirectory() as tmp:
        h = C.c_void_p()
        _lib.check(lib.selm_dcd_open_sim(os.path.join(tmp, "t.dcd").encode(), sim._h, 1, C.byref(h)))
        t0 = time.perf_counter()
        for _ in range(frames):
            _lib.check(lib.selm_dcd_write_sim(h, sim._h))
        frame_ms = 1e3 * (time.perf_counter() - t0) / frames
        _lib.check(lib.selm_dcd_close(h))
    return {"analysis_sample_us": round(sample_us, 2), "analysis": "MSD 40 lags (ring of 41 float32 frames), "
            "S(q) at 16 wavevectors, K_d; device time per sample", "dcd_frame_ms": round(frame_ms, 3),
            "dcd": "one frame of 1e5 monomers: device read-back plus the file write (host)"}


def cpu_baseline(wl, budget_s=15.0):
    """The reference's own CPU code (oracle/_ref; else the FP64 oracle port)
    on all the host's hardware threads, one single-rank instance of the same
    workload per thread, as the reference arm runs it: a bounded sample of
    about `budget_s` seconds (a step takes about 1 s per instance at 128^3
    with 1e5 monomers)."""
    kind = reference_kind()
    workers = reference_workers()
    steps = max(2, int(budget_s))
    value, window = time_reference(wl, kind, 1, steps, workers)
    what = "the reference's own CPU code" if kind == "reference" else "FP64 oracle port"
    return {"value": value, "unit": "fluid-cell-steps/s", "cores": workers, "kind": kind,
            "sample": f"{workers} concurrent single-rank instances x {steps} full steps of the same workload "
                      f"({what}), {window:.1f} s from the first start to the last end"}


def fp32_accuracy(wl, stream, marks=(1, 10, 100)):
    """Relative velocity error of the FP32 fused form against the FP64 fused
    form (which matches the reference's own code to 1e-12 per step) on the
    headline workload, both started from the same state: monomer velocities
    and the fluid velocity, each as max |v32 - v64| / max |v64|, after
    `marks` steps; at kT = 1 (same Philox stream) and at kT = 0 with a body
    force of 0.01.  Step 1 is the error of one step; later marks add the
    growth of a chaotic trajectory (WCA collisions amplify any difference)."""
    from dataclasses import replace

    from monomers2026_b200.selm import Selm

    def rel(a, b):
        s = np.abs(b).max()
        return float(np.abs(a - b).max() / (s if s > 0 else 1.0))

    out = {}
    topo0 = replace(wl.topology, body_force=(0.01, 0.0, 0.0))
    cases = (("kT1", wl.params, wl.topology),
             ("kT0_body", replace(wl.params, T=0.0, flagStochasticDriving=0), topo0))
    for tag, prm, topo in cases:
        sims = []
        for form in ("fused64", "fused32"):
            s = Selm(replace(prm, form=form, integrator="inertial"), wl.x, wl.mass, topology=topo)
            s.set_stream(stream.cuda_stream)
            s.initial()
            sims.append(s)
        rows = {"steps": list(marks), "v": [], "u": []}
        done = 0
        for m in marks:
            for s in sims:
                s.run(m - done)
            done = m
            (_, v64, _), (_, v32, _) = sims[0].particles(), sims[1].particles()
            rows["v"].append(rel(v32, v64))
            rows["u"].append(rel(sims[1].get_field(0), sims[0].get_field(0)))
        for s in sims:
            s.final()
        out[tag] = rows
    out["one_step_max"] = max(max(out[t]["v"][0], out[t]["u"][0]) for t in ("kT1", "kT0_body"))
    return out


def reference_gpu_baseline(wl, kern, steps=10):
    """The reference's own GPU step (oracle/_ref/libselm_refgpu.so: its
    cuda/SELM_Eulerian_Period.cu and cuda/SELM_Kernel.cu built unchanged for
    sm_100a with a stub driver) on the same workload, the host LAMMPS force
    call left out (the conservative force is held at zero), per phase with
    CUDA events; and cuFFT's batched R2C + C2R of the three 128^3 fields
    (FP32 and FP64) beside this library's three fluid kernels, whose FFTs
    carry the spectral update as well.  A baseline, like cpu_baseline: not
    part of this library's step."""
    from oracle import refgpu
    if not refgpu.available():
        return None, None
    n = wl.params.numMeshPtsPerDir[0]
    r = refgpu.ReferenceGpuRun(wl)
    r.step(3)
    t = r.time(steps)
    r.close()
    N = n ** 3
    ref = {"ms_per_step": t["step"], "kernels_ms": {k: round(v, 4) for k, v in t.items() if k != "step"},
           "value": N / (t["step"] / 1e3), "unit": "fluid-cell-steps/s", "steps": steps,
           "what": "reference cuda/ step (lagrangian_update with FP64 atomics, cuFFT D2Z/Z2D projection, "
                   "CUB mean removal, cuRAND + cuFFT thermal forcing), host LAMMPS forces left out"}
    fl = sum(kern.get(k, (0.0, 0))[0] for k in ("xy_forward", "z_update", "xy_inverse"))
    x32 = refgpu.cufft_time(n, 32)
    x64 = refgpu.cufft_time(n, 64)
    xc = {"grid": n, "fields": 3,
          "cufft_fp32_ms": {k: round(v, 4) for k, v in x32.items()},
          "cufft_fp64_ms": {k: round(v, 4) for k, v in x64.items()},
          "cufft_fp32_r2c_plus_c2r_ms": round(x32["r2c_ms"] + x32["c2r_ms"], 4),
          "own_fluid_kernels_ms": round(fl, 4),
          "note": "own = xy forward + z update (z FFTs, spectral update, noise) + xy inverse of the headline form"}
    return ref, xc


# --------------------------------------------------------------------------- reference arm
# Resident memory of one single-rank reference instance of the 128^3 workload
# with 1e5 monomers (measured 0.37 GB) plus its interpreter, rounded up.
REF_INSTANCE_BYTES = 0.75e9


def _host_memory_available() -> float:
    """Bytes this process may still allocate: the smaller of the host's
    available memory and what its memory cgroup (v2 or v1) leaves."""
    import psutil
    avail = float(psutil.virtual_memory().available)
    for lim, use in (("/sys/fs/cgroup/memory.max", "/sys/fs/cgroup/memory.current"),
                     ("/sys/fs/cgroup/memory/memory.limit_in_bytes", "/sys/fs/cgroup/memory/memory.usage_in_bytes")):
        try:
            with open(lim) as f:
                t = f.read().strip()
            if t == "max":
                continue
            with open(use) as f:
                avail = min(avail, float(t) - float(f.read().strip()))
        except (OSError, ValueError):
            continue
    return avail


def reference_workers(limit: int | None = None) -> int:
    """Concurrent single-rank instances the host runs: one per usable hardware
    thread, no more than half the available memory holds."""
    cpus = len(os.sched_getaffinity(0))
    by_mem = int(0.5 * _host_memory_available() // REF_INSTANCE_BYTES)
    n = max(1, min(cpus, by_mem))
    return min(n, limit) if limit else n


def reference_kind() -> str:
    """"reference" when the reference's own CPU source is built under
    oracle/_ref, else "port" (the FP64 oracle restatement)."""
    try:
        from oracle import refdriver
        return "reference" if refdriver.available() else "port"
    except Exception:
        return "port"


def _reference_instance(wl, kind):
    p = wl.params
    if kind == "reference":
        from oracle import refdriver
        return refdriver.ReferenceRun(wl)
    from oracle import pyoracle as O
    ff = O.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    run = O.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass,
                stochastic=p.flagStochasticDriving, seed=p.SELM_Seed, ff=ff)
    run.initial()
    return run


def _reference_worker(wl, kind, warmup, steps, barrier, results, i):
    """One instance in its own process: warm up, wait for all, time `steps`
    full steps.  Its stdout goes to /dev/null (one JSON line from the parent)."""
    try:
        fd = os.open(os.devnull, os.O_WRONLY)
        os.dup2(fd, 1)
        run = _reference_instance(wl, kind)
        for _ in range(warmup):
            run.step(1)
        barrier.wait()
        t0 = time.perf_counter()
        for _ in range(steps):
            run.step(1)
        results.put((i, t0, time.perf_counter(), ""))
    except Exception as e:  # reported by the parent
        barrier.abort()
        results.put((i, 0.0, 0.0, f"{type(e).__name__}: {e}"))


def time_reference(wl, kind, warmup, steps, workers, timeout_s=1800.0):
    """Aggregate rate of `workers` concurrent instances of the same workload:
    (instances x steps x cells) / (last end - first start).  CLOCK_MONOTONIC
    (perf_counter) is one clock for all processes of the host."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers, timeout=timeout_s)
    results = ctx.Queue()
    procs = [ctx.Process(target=_reference_worker, args=(wl, kind, warmup, steps, barrier, results, i), daemon=True)
             for i in range(workers)]
    for q in procs:
        q.start()
    got, err, done = [], [], set()
    deadline = time.time() + timeout_s
    while len(done) < workers and not err:
        try:
            i, t0, t1, e = results.get(timeout=2.0)
            done.add(i)
            (err if e else got).append(e if e else (t0, t1))
        except Exception:
            dead = [k for k, q in enumerate(procs) if k not in done and q.exitcode not in (None, 0)]
            if dead:
                err.append(f"instance {dead[0]} exited with code {procs[dead[0]].exitcode}")
            elif time.time() > deadline:
                err.append("no result before the deadline")
    if err:
        barrier.abort()
    for q in procs:
        q.join(timeout=30)
        if q.is_alive():
            q.kill()
    if err:
        raise RuntimeError("reference instance failed: " + err[0])
    window = max(t1 for _, t1 in got) - min(t0 for t0, _ in got)
    N = int(np.prod(wl.params.numMeshPtsPerDir))
    return N * workers * steps / window, window


def run_reference(args, rank, world):
    if rank != 0:
        return
    from monomers2026_b200 import workloads as W
    wl = W.config(3)
    p = wl.params
    N = int(np.prod(p.numMeshPtsPerDir))
    kind = reference_kind()
    what = ("the reference's own CPU code (mpi/ sources, single rank each)" if kind == "reference"
            else "the FP64 oracle port (single thread each)")
    workers = reference_workers(args.ref_workers)
    value, window = time_reference(wl, kind, args.warmup, args.steps, workers)
    out = {
        "impl": "reference",
        "metric": "fluid-cell-steps/s @128^3, 1e5 monomers (FP32 fused form; plain FP64 form beside it)",
        "value": value, "unit": "fluid-cell-steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": N / value * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded random-walk FENE chains)",
        "config": headline_config(p.numMeshPtsPerDir[0], len(wl.mass), world),
        "form": "the reference's CPU step (FP64)" if kind == "reference" else "FP64 oracle port",
        "cpu_baseline": {"value": value, "unit": "fluid-cell-steps/s", "cores": workers, "kind": kind,
                         "sample": f"{workers} concurrent instances x {args.steps} full steps of the same workload "
                                   f"through {what}, one per host thread; value = all their cell-steps over "
                                   f"the {window:.1f} s from the first start to the last end"},
        "e2e": {"value": value, "unit": "fluid-cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="fused32", choices=["fused32", "fused64", "plain64"])
    ap.add_argument("--no-forms", action="store_true", help="skip timing the other forms")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--ref-workers", type=int, default=None,
                    help="reference arm: cap on concurrent instances (default: one per host thread)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-ensemble and serving runs")
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--no-autotune", action="store_true", help="keep the built-in kernel choices")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
