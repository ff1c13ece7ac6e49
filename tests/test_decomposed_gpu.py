"""The decomposed instance (z slabs over ranks) on one GPU: every rank's slab
in this process, exchanging through the loopback transport, against the
whole instance on the same inputs.  The slabs run the whole instance's
kernels on their parts (the spread of a slab's tiles, the FFTs of its
planes, the z pass of its columns); only the interpolation is summed slab by
slab.  So one rank is bitwise the whole instance (FP32 with the multi-filing
spread, below 16384 monomers), the FP64 form agrees to 1e-12 per step
(positions, velocities, forces, fluid velocity; relative to each field's
maximum) and the FP32 form to 1e-5, at kT = 0 and kT = 1 (same Philox
stream), including the bench workload (128^3, 1e5 FENE monomers) over 8
slabs."""
from dataclasses import replace

import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.decomposed import Decomposed, LoopbackTransport
from monomers2026_b200.selm import Selm

pytestmark = pytest.mark.gpu


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def _pair(wl, form, R, v0):
    p = replace(wl.params, form=form)
    whole = Selm(p, wl.x, wl.mass, v=v0, topology=wl.topology)
    whole.initial()
    dec = Decomposed(p, wl.x, wl.mass, v=v0, topology=wl.topology, transport=LoopbackTransport(R))
    dec.initial()
    return whole, dec


def _fields(whole, dec):
    x, v, f = whole.particles()
    xd, vd, fd = dec.particles()
    u = whole.get_field(0)
    ud = np.concatenate([a for _, a in sorted(dec.velocity().items())], axis=1)
    return (x, v, f, u), (xd, vd, fd, ud)


def _compare(wl, form, R, steps, tol, v0=None):
    whole, dec = _pair(wl, form, R, v0)
    worst = 0.0
    for k in range(steps):
        whole.run(1)
        dec.step(1)
        a, b = _fields(whole, dec)
        errs = [rel(q, p) for p, q in zip(a, b)]
        assert max(errs) <= tol, f"step {k + 1}: x v f u {errs}"
        worst = max(worst, max(errs))
    assert dec.status() == whole.status() == 0
    whole.final()
    dec.final()
    return worst


def test_one_slab_is_the_whole_instance_bitwise():
    wl = W.config(1, kT=1.0, grid=32, nchains=12, length=20)
    v0 = np.random.default_rng(2).normal(0.0, 0.3, wl.x.shape)
    assert _compare(wl, "fused32", 1, 4, 0.0, v0) == 0.0


@pytest.mark.parametrize("kT", [0.0, 1.0])
def test_two_slabs_fp64(kT):
    wl = W.config(1, kT=kT, grid=32, nchains=12, length=20)
    wl.params.flagStochasticDriving = int(kT > 0)
    v0 = np.random.default_rng(3).normal(0.0, 0.3, wl.x.shape)
    _compare(wl, "fused64", 2, 6, 1e-12, v0)


def test_four_slabs_fene_fp32_and_fp64():
    wl = W.config(2, kT=1.0, nchains=10, length=100)  # 64^3, FENE + WCA chains
    _compare(wl, "fused64", 4, 4, 1e-12)
    _compare(wl, "fused32", 4, 4, 1e-5)


def test_bench_workload_over_eight_slabs_fp32():
    wl = W.config(3, form="fused32", seed=1003)  # 128^3, 1e5 FENE + WCA monomers, kT = 1
    _compare(wl, "fused32", 8, 3, 1e-5)


def _nccl_one_rank(port, q):
    import datetime
    import os

    import torch
    import torch.distributed as dist

    from monomers2026_b200.decomposed import TorchTransport
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        wl = W.config(1, kT=1.0, grid=32, nchains=12, length=20)
        v0 = np.random.default_rng(2).normal(0.0, 0.3, wl.x.shape)
        p = replace(wl.params, form="fused32")
        whole = Selm(p, wl.x, wl.mass, v=v0, topology=wl.topology)
        whole.initial()
        whole.run(3)
        dec = Decomposed(p, wl.x, wl.mass, v=v0, topology=wl.topology, transport=TorchTransport())
        dec.initial()
        dec.step(3)
        a, b = _fields(whole, dec)
        q.put(("ok", [float(np.abs(x - y).max()) for x, y in zip(a, b)], dec.status()))
        whole.final()
        dec.final()
    except Exception as e:  # reported to the test
        q.put(("error", repr(e), -1))
    finally:
        dist.destroy_process_group()


def test_nccl_transport_one_rank_is_the_whole_instance():
    """The torch.distributed transport on NCCL (all_reduce, all_to_all) with
    one rank, in a child process: bitwise the whole instance."""
    import socket

    import torch.multiprocessing as mp

    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=_nccl_one_rank, args=(port, q))
    proc.start()
    kind, errs, status = q.get(timeout=300)
    proc.join(timeout=60)
    assert kind == "ok", errs
    assert errs == [0.0, 0.0, 0.0, 0.0] and status == 0
