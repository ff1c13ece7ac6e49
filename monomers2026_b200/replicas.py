"""Replica sharding across ranks (one process per GPU).

The SELM step has no exchange between independent simulations, so multi-GPU
runs are replicas: every rank owns a disjoint set of jobs, steps them with no
data-path collective, and the only communication is the barrier and the
max-over-ranks reduction of the timing.  These helpers are the host logic of
that scheme; they work with any torch.distributed backend (NCCL on GPUs, gloo
on CPU for tests).
"""
from __future__ import annotations

from dataclasses import dataclass


def replica_seed(base_seed: int, rank: int) -> int:
    """Philox key of the replica a rank runs (distinct per rank, stable across runs)."""
    return int(base_seed) + int(rank)


def shard_jobs(costs, world: int):
    """Assign jobs (by estimated cost, e.g. grid points x steps) to ranks.

    Longest-processing-time-first greedy: jobs sorted by decreasing cost, each
    to the currently least-loaded rank (ties to the lowest rank), so the
    assignment is deterministic.  Returns a list of job-index lists per rank."""
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    out = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += float(costs[i])
    for lst in out:
        lst.sort()
    return out


@dataclass
class StepTiming:
    total_ms: float
    steps: int


def max_over_ranks(value: float, device=None) -> float:
    """Max of a per-rank float over the default process group (identity when not initialised)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: float, world: int, max_seconds: float) -> float:
    """Aggregate throughput: units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / max_seconds
