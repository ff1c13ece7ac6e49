"""Autotuner for the fused forms: picks the four-step FFT split and the
z-kernel occupancy per (grid size, precision) by timing them.

For one representative workload of a shape, ``tune`` creates a throwaway
simulation, times a few steps of every candidate configuration on the device
(CUDA events, L2 flushed between steps), and records the fastest with
``selm_tune_default`` so that every simulation of that shape created later in
the process starts from it.  The simulations being served are never stepped
for tuning.  ``tune_ensemble`` does this once per distinct shape of a list of
workloads (the batched ensemble mixes several grid sizes).
"""
from __future__ import annotations

import itertools

from .selm import TUNE_FFT_SPLIT, TUNE_Z_BLOCKS, Selm, tune_default

SPLITS = (0, 1)
Z_BLOCKS = (0, 2, 3, 4)


def _time_steps(sim: Selm, stream, steps: int, flush) -> float:
    import torch

    best = float("inf")
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.run(1)
        b.record(stream)
        b.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def four_step_splits(n: int) -> tuple:
    """N1 of the default (largest factor <= 16) and of the most balanced
    four-step split of a line length n (N2 = n / N1 <= 16), as in the kernels."""
    default = next((a for a in range(16, 0, -1) if n % a == 0 and n // a <= a), 0)
    balanced = min((a for a in range(1, 17) if n % a == 0 and n // a <= 16 and a >= n // a), default=0)
    return default, balanced


def tune(workload, steps: int = 6, warmup: int = 2, splits=SPLITS, z_blocks=Z_BLOCKS, record: bool = True) -> dict:
    """Time every (split, z blocks) candidate on a throwaway copy of ``workload``
    (fused forms); returns {"choice": {...}, "ms": {...}} and, when ``record``,
    makes the choice the default for this grid size and precision."""
    import torch

    p = workload.params
    n = int(p.numMeshPtsPerDir[0])
    prec = 32 if p.form == "fused32" else 64
    d, b = four_step_splits(n)
    if d == b:  # one split for this size
        splits = tuple(x for x in splits if x == 0) or (0,)
    sim = Selm(p, workload.x, workload.mass, v=workload.v, topology=workload.topology)
    sim.initial()
    stream = torch.cuda.Stream()
    sim.set_stream(stream.cuda_stream)
    flush = torch.empty(32 << 20, dtype=torch.float32, device="cuda")
    timings = {}
    for split, zb in itertools.product(splits, z_blocks):
        sim.tune(TUNE_FFT_SPLIT, split)
        sim.tune(TUNE_Z_BLOCKS, zb)
        sim.run(warmup)
        timings[(split, zb)] = _time_steps(sim, stream, steps, flush)
    sim.final()
    (split, zb), ms = min(timings.items(), key=lambda kv: kv[1])
    if record:
        tune_default(n, prec, TUNE_FFT_SPLIT, split)
        tune_default(n, prec, TUNE_Z_BLOCKS, zb)
    return {"grid": n, "precision": prec, "choice": {"fft_split": split, "z_blocks_per_sm": zb},
            "ms": {f"split{k[0]}_z{k[1]}": round(v, 4) for k, v in timings.items()}}


def tune_ensemble(workloads, **kw) -> list:
    """Tune once per distinct (grid size, form) of ``workloads``, on the
    replica with the most monomers of that shape."""
    by_shape = {}
    for w in workloads:
        key = (int(w.params.numMeshPtsPerDir[0]), w.params.form)
        if key not in by_shape or len(w.mass) > len(by_shape[key].mass):
            by_shape[key] = w
    return [tune(w, **kw) for _, w in sorted(by_shape.items())]
