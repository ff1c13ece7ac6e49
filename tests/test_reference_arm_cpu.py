"""The reference arm of bench.py on CPU: single-rank instances of one
workload run concurrently, one per host thread, and timed over the window
from the first start to the last end."""
import dataclasses
import os

import pytest


def test_reference_workers_bounds():
    import bench
    n = bench.reference_workers()
    assert 1 <= n <= len(os.sched_getaffinity(0))
    assert bench.reference_workers(1) == 1
    assert bench._host_memory_available() > 0


def test_concurrent_port_instances(oracle):
    import bench
    from monomers2026_b200 import workloads as W
    wl = W.config(1)
    rate, window = bench.time_reference(wl, "port", warmup=1, steps=2, workers=2, timeout_s=300)
    N = 32 ** 3
    assert window > 0 and rate == pytest.approx(N * 2 * 2 / window)


def test_failed_instance_is_reported(oracle):
    """An instance that raises before the common start aborts the barrier:
    the others stop and the parent raises instead of waiting."""
    import bench
    from monomers2026_b200 import workloads as W
    wl = dataclasses.replace(W.config(1), topology=None)
    with pytest.raises(RuntimeError, match="reference instance failed"):
        bench.time_reference(wl, "port", warmup=1, steps=1, workers=2, timeout_s=300)
