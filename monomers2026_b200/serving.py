"""Batched ensembles and a continuous-batching server on one GPU.

The reference runs one simulation per process.  Here many simulations of
the fused forms live on the device at once and step together, one CUDA-graph
launch per step (``Batch``):

* ``run_ensemble`` steps a fixed set of replicas (the batched-ensemble
  configuration) and reports replica-steps/s and the per-step latency of
  the batch launch (CUDA events on the batch stream, p50/p99);
* ``run_sequential`` steps the same replicas one after another with single
  launches (the plain FP64 form for the reference-structured baseline);
* ``Server`` admits jobs as they arrive while their device memory fits an
  HBM budget, adds them to the running batch between steps, and retires each
  job when its steps are done (state read back, memory freed): continuous
  batching.  A job's result does not depend on what else is in the batch
  (each member keeps its own buffers and Philox counters).  The host stays
  off the step's critical path: simulations are created on a worker thread
  while the batch steps, a job carries its step budget into the batch
  (selm_batch_add_job), finished jobs are found by an event query
  (selm_batch_poll) and read back on their own stream (selm_batch_retire),
  and device memory comes from the library's stream-ordered pool, so neither
  creation nor release waits for the batch.
"""
from __future__ import annotations

import dataclasses
import math
import queue as _queue
import threading
import time
from collections import deque

import numpy as np

from .selm import Batch, Selm

_FP = {"fused32": 4, "fused64": 8, "plain64": 8}
SPREAD_TILE = (16, 8, 16)  # cells of a spread tile (kTX, kTY, kTZ of the engine)
HOME_MIN_MONOMERS = 16384  # FP32 simulations with at least this many monomers spread by home tiles


def estimate_device_bytes(params, natoms: int, pairs: bool = True) -> int:
    """Upper estimate of the device memory of one simulation (for admission
    before it is created): fields, spectra, monomer arrays (with the staging
    buffers of a per-step upload), stencil records, tile and force-cell
    buckets and the neighbour list."""
    nx, ny, nz = (int(v) for v in params.numMeshPtsPerDir)
    N = nx * ny * nz
    N2 = (nx // 2 + 1) * ny * nz
    s = _FP[params.form]
    if params.form == "plain64":
        grid = 8 * (3 * N * 4 + N * 3) + 16 * 3 * N2
    else:
        grid = 2 * 3 * N * s + 2 * 3 * N2 * 2 * s
    tile = SPREAD_TILE
    nb = [-(-n // t) for n, t in zip((nx, ny, nz), tile)]
    tiles = nb[0] * nb[1] * nb[2]
    M = max(1, int(natoms))
    # FP32 grids with at least HOME_MIN_MONOMERS: one filing per monomer, plus the tiles' halo boxes
    home = params.form == "fused32" and M >= HOME_MIN_MONOMERS
    per = 1.0
    if not home:
        for b, t in zip(nb, tile):
            per *= 1.0 if b == 1 else 1.0 + 4.0 / t
    cap = max(128, -(-(int(math.ceil(4.0 * M * per / tiles)) + 64) // 32) * 32)
    slots = 4 * tiles * (cap + 1) + 8 * ((1 if home else 27) * M + 1024)  # tile slots and the overflow list
    if home:
        slots += tiles * (4 * 3 * (tile[0] + 4) * (tile[1] + 4) * (tile[2] + 4) + 16)
    # x (two buffers), v, f, tf, m, the staged upload of a per-step round trip, stencil records
    mono = M * (2 * 24 + 3 * 24 + 8 + 2 * 24 + (128 if s == 4 else 224)) + slots
    nl = 0
    if pairs:
        nc3 = min(2 * M, N) + 1
        nl = 4 * (64 * M + 2 * M) + 24 * M + 4 * (4 * nc3 + 4 * M)
    return int(1.1 * (grid + mono + nl)) + (1 << 20)


def _make(wl, form=None) -> Selm:
    p = wl.params
    if form is not None:
        p = dataclasses.replace(p, form=form)
    s = Selm(p, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    s.initial()
    return s


def _pcts(ms):
    a = np.asarray(ms, dtype=float)
    return {"p50": float(np.percentile(a, 50)), "p99": float(np.percentile(a, 99)), "mean": float(a.mean())}


def run_ensemble(workloads, steps: int, warmup: int = 3, form: str = "fused32"):
    """Step all replicas together; device-timed per batch launch."""
    import torch

    sims = [_make(w, form) for w in workloads]
    b = Batch()
    for s in sims:
        b.add(s)
    stream = torch.cuda.ExternalStream(b.stream)
    b.run(warmup)
    b.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for a, e in ev:
        a.record(stream)
        b.run(1)
        e.record(stream)
    b.synchronize()
    per = [a.elapsed_time(e) for a, e in ev]
    total_ms = float(sum(per))
    cells = sum(int(np.prod(w.params.numMeshPtsPerDir)) for w in workloads)
    status = [s.status() for s in sims]
    out = {
        "replicas": len(sims),
        "steps": steps,
        "replica_steps_per_s": len(sims) * steps / (total_ms / 1e3),
        "cell_steps_per_s": cells * steps / (total_ms / 1e3),
        "step_ms": _pcts(per),
        "device_bytes": int(sum(s.device_bytes() for s in sims)),
        "status_nonzero": int(sum(1 for w in status if w)),
    }
    b.final()
    for s in sims:
        s.final()
    return out


def run_sequential(workloads, steps: int, form: str = "plain64"):
    """Each replica stepped alone, one after another (device-timed per replica)."""
    import torch

    total_ms = 0.0
    for w in workloads:
        s = _make(w, form)
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        s.run(1)
        s.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.run(steps)
        e.record(st)
        e.synchronize()
        total_ms += a.elapsed_time(e)
        s.final()
    return {"replicas": len(workloads), "steps": steps,
            "replica_steps_per_s": len(workloads) * steps / (total_ms / 1e3)}


def run_sequential_jobs(jobs, form: str = "plain64", sample_steps: int = 10):
    """The serving jobs run one after another, each alone in ``form``: every
    job's step is device-timed over ``sample_steps`` steps (after one
    untimed step) and counted for all of its ``nsteps``.  Returns the
    replica-steps/s of that sequence (creation and read-back not counted)."""
    import torch

    total_ms = 0.0
    steps = 0
    for j in jobs:
        s = _make(j.workload, form)
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        s.run(1)
        s.synchronize()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(st)
        s.run(sample_steps)
        e.record(st)
        e.synchronize()
        total_ms += a.elapsed_time(e) / sample_steps * j.nsteps
        steps += j.nsteps
        s.final()
    return {"jobs": len(jobs), "sample_steps": sample_steps, "replica_steps_per_s": steps / (total_ms / 1e3)}


@dataclasses.dataclass
class Job:
    jid: int
    workload: object
    nsteps: int
    arrival: float  # seconds after the start of the run
    admitted: float = math.nan
    done: float = math.nan
    x: np.ndarray | None = None
    v: np.ndarray | None = None
    status: int = 0
    est_bytes: int = 0
    left: int = 0  # batch steps still to take


class Server:
    """Continuous batching under an HBM budget.

    ``run(jobs)`` plays the arrivals on the wall clock: between two batch
    steps it admits every arrived job whose estimated memory fits the budget
    (first come, first served), then steps the batch once; jobs whose steps
    are done are read back and retired, freeing their memory for the queue.
    When every admitted job has taken its steps and only their read-backs
    are outstanding, the loop waits for those instead of stepping an empty
    batch; the per-step latencies are those of steps with work."""

    AHEAD = 3  # batch steps in flight at most

    def __init__(self, budget_bytes: int, form: str = "fused32"):
        self.budget = int(budget_bytes)
        self.form = form
        self.used = 0
        self.peak = 0
        self.batch = Batch()

    def run(self, jobs: list[Job], max_seconds: float = 600.0):
        import torch

        stream = torch.cuda.ExternalStream(self.batch.stream)
        dev = torch.cuda.current_device()
        pending = deque(sorted(jobs, key=lambda j: j.arrival))
        waiting: deque = deque()  # arrived, not yet admitted
        todo: _queue.Queue = _queue.Queue()  # admitted: created by the worker
        ready: _queue.Queue = _queue.Queue()  # (job, sim or exception)
        creating = 0
        active: dict = {}  # sim handle -> (job, sim)
        step_ev = []
        finished = []

        def worker():
            torch.cuda.set_device(dev)
            while True:
                j = todo.get()
                if j is None:
                    return
                try:
                    ready.put((j, _make(j.workload, self.form)))
                except Exception as e:  # reported by the loop
                    ready.put((j, e))

        th = threading.Thread(target=worker, daemon=True)
        th.start()
        t0 = time.perf_counter()
        try:
            while pending or waiting or creating or active:
                now = time.perf_counter() - t0
                if now > max_seconds:
                    raise RuntimeError("serving run exceeded its time bound")
                while pending and pending[0].arrival <= now:
                    waiting.append(pending.popleft())
                # admission by the HBM budget, first come first served; creation on the worker
                while waiting:
                    j = waiting[0]
                    est = estimate_device_bytes(dataclasses.replace(j.workload.params, form=self.form),
                                                len(j.workload.mass))
                    if self.used + est > self.budget and (active or creating):
                        break
                    waiting.popleft()
                    self.used += est
                    self.peak = max(self.peak, self.used)
                    j.est_bytes = est
                    creating += 1
                    todo.put(j)
                # jobs created since the last step join the batch with their budgets
                while True:
                    try:
                        j, s = ready.get_nowait()
                    except _queue.Empty:
                        break
                    creating -= 1
                    if isinstance(s, Exception):
                        raise s
                    self.batch.add_job(s, j.nsteps)
                    j.left = j.nsteps
                    j.admitted = time.perf_counter() - t0
                    active[s._h.value] = (j, s)
                if not active:
                    time.sleep(0.0005)
                    continue
                stepping = [j for j, _ in active.values() if j.left > 0]
                if stepping:
                    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    self.batch.run(1)
                    e.record(stream)
                    step_ev.append((a, e, len(stepping)))
                    for j in stepping:
                        j.left -= 1
                    # at most AHEAD steps in flight: the host does not queue
                    # seconds of work ahead of the device, which kept the
                    # creation of new jobs waiting behind the batch's streams
                    if len(step_ev) > self.AHEAD:
                        step_ev[-1 - self.AHEAD][1].synchronize()
                # finished jobs: an event query, then a read-back on the job's own stream
                retired = self.batch.poll()
                for s in retired:
                    j, _ = active.pop(s._h.value)
                    j.x, j.v, _f = self.batch.retire(s)
                    j.status = s.status()
                    j.done = time.perf_counter() - t0
                    s.final()
                    self.used -= j.est_bytes
                    finished.append(j)
                if not stepping and not retired:
                    time.sleep(0.0002)  # only read-backs outstanding
        finally:
            todo.put(None)
            th.join(timeout=30)
        self.batch.synchronize()
        per = [a.elapsed_time(e) for a, e, _ in step_ev]
        wall = time.perf_counter() - t0
        rs = sum(j.nsteps for j in finished)
        cells = sum(int(np.prod(j.workload.params.numMeshPtsPerDir)) * j.nsteps for j in finished)
        return {
            "jobs": len(finished),
            "batch_steps": len(per),
            "max_batch": max((n for _, _, n in step_ev), default=0),
            "step_ms": _pcts(per) if per else None,
            "job_latency_s": _pcts([j.done - j.arrival for j in finished]),
            "replica_steps_per_s_device": rs / (sum(per) / 1e3) if per else 0.0,
            "replica_steps_per_s_wall": rs / wall,
            "cell_steps_per_s_device": cells / (sum(per) / 1e3) if per else 0.0,
            "peak_device_bytes": int(self.peak),
            "wall_s": wall,
            "status_nonzero": sum(1 for j in finished if j.status),
        }

    def final(self):
        self.batch.final()


def serving_jobs(njobs: int, rate: float = 200.0, grids=(32, 48, 64, 96, 128),
                 weights=(0.3, 0.3, 0.2, 0.15, 0.05), m_range=(20, 5000), steps_range=(500, 5000),
                 steps_scale: float = 1.0, seed: int = 1005, form: str = "fused32") -> list[Job]:
    """Serving configuration: Poisson arrivals at ``rate``/s, grid by ``weights``,
    one chain of U[m_range] monomers, U[steps_range] steps (times
    ``steps_scale`` for a bounded run), kT in [0.5, 2]; job j has geometry and
    Philox seed ``seed * 1000 + j``."""
    from .workloads import replica

    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for jid in range(njobs):
        t += rng.exponential(1.0 / rate)
        n = int(rng.choice(grids, p=np.asarray(weights) / np.sum(weights)))
        M = int(rng.integers(m_range[0], m_range[1] + 1))
        steps = max(1, int(round(rng.integers(steps_range[0], steps_range[1] + 1) * steps_scale)))
        kT = float(rng.uniform(0.5, 2.0))
        wl = replica(n, 1, M, kT, seed * 1000 + jid, form=form)
        jobs.append(Job(jid=jid, workload=wl, nsteps=steps, arrival=t))
    return jobs
