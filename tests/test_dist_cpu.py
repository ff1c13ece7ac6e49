"""Multi-rank host logic on CPU (gloo, world size 2): replica seeds, job
sharding and the max-over-ranks timing used by bench.py --gpus N."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from monomers2026_b200.replicas import replica_seed, shard_jobs, whole_job_rate


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    from monomers2026_b200.replicas import max_over_ranks
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 10.0 + 5.0 * rank
        m = max_over_ranks(local_ms)
        jobs = shard_jobs([5, 1, 4, 4, 2, 7], world)[rank]
        t = torch.tensor([len(jobs)], dtype=torch.int64)
        dist.all_reduce(t)
        q.put((rank, m, replica_seed(1003, rank), jobs, int(t.item())))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]  # both ranks see the slowest rank's time
    assert res[0][2] != res[1][2]  # distinct replica seeds
    assert sorted(res[0][3] + res[1][3]) == list(range(6))  # disjoint shards covering all jobs
    assert res[0][4] == 6


def test_sharding_is_balanced_and_deterministic():
    costs = [128 ** 3] * 3 + [32 ** 3] * 20 + [96 ** 3] * 5
    a = shard_jobs(costs, 4)
    assert a == shard_jobs(costs, 4)
    loads = [sum(costs[i] for i in s) for s in a]
    assert max(loads) / min(loads) < 1.5
    assert whole_job_rate(100.0, 4, 2.0) == 200.0


@pytest.mark.parametrize("world", [1, 3])
def test_sharding_covers_every_job_once(world):
    s = shard_jobs(list(range(17)), world)
    assert sorted(i for r in s for i in r) == list(range(17))
