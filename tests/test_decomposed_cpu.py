"""Exchange logic of the decomposed instance on CPU: the slab layout, and the
two all-to-alls (z slabs of the xy spectrum to blocks of half-spectrum
columns and back) and the summed interpolation, through gloo ranks (world
sizes 2 and 4) and the in-process loopback transport.  Each rank's slab of a
seeded [3][n][ncol] array goes through the exchanges and must arrive as
exactly the columns the layout gives that rank, and come back unchanged."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from monomers2026_b200.decomposed import (LoopbackTransport, SlabLayout, pack_to_columns, pack_to_planes,
                                          recv_buffers, unpack_columns, unpack_planes)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _global(lay: SlabLayout, dtype=torch.float64):
    g = torch.Generator().manual_seed(7)
    return torch.randn((3, lay.n, lay.ncol, 2), generator=g, dtype=dtype)


@pytest.mark.parametrize("n,R", [(16, 1), (32, 2), (48, 3), (64, 4)])
def test_layout_covers_planes_and_columns_once(n, R):
    lay = SlabLayout(n, R)
    planes = [z for r in range(R) for z in range(lay.planes(r)[0], sum(lay.planes(r)))]
    cols = [c for r in range(R) for c in range(lay.cols(r)[0], sum(lay.cols(r)))]
    assert planes == list(range(n)) and cols == list(range(lay.ncol))


def _exchange_round(lay, T, works):
    """Forward and back exchange of the slabs in `works` (one per local rank)."""
    bufs = [recv_buffers(lay, r, w) for r, w in zip(T.local, works)]
    cols = [torch.zeros((3, lay.n, lay.cols(r)[1], 2), dtype=w.dtype) for r, w in zip(T.local, works)]
    T.alltoall([pack_to_columns(w, lay) for w in works], [b[0] for b in bufs])
    for b, c in zip(bufs, cols):
        unpack_columns(b[0], c, lay)
    back = [torch.zeros_like(w) for w in works]
    T.alltoall([pack_to_planes(c, lay) for c in cols], [b[1] for b in bufs])
    for b, w in zip(bufs, back):
        unpack_planes(b[1], w, lay)
    return cols, back


def _check(lay, ranks, cols, back, full):
    for r, c, w in zip(ranks, cols, back):
        c0, ncl = lay.cols(r)
        z0, nzl = lay.planes(r)
        assert torch.equal(c, full[:, :, c0:c0 + ncl])  # this rank's columns, every plane
        assert torch.equal(w, full[:, z0:z0 + nzl])  # the round trip returns the slab unchanged


@pytest.mark.parametrize("n,R", [(32, 2), (48, 3), (64, 4)])
def test_loopback_exchanges(n, R):
    lay = SlabLayout(n, R)
    full = _global(lay)
    T = LoopbackTransport(R)
    works = [full[:, lay.planes(r)[0]:sum(lay.planes(r))].clone() for r in range(R)]
    cols, back = _exchange_round(lay, T, works)
    _check(lay, range(R), cols, back, full)
    bufs = [torch.full((6,), float(r + 1), dtype=torch.float64) for r in range(R)]
    T.allreduce_sum(bufs)
    assert all(torch.equal(b, torch.full((6,), R * (R + 1) / 2, dtype=torch.float64)) for b in bufs)


def _worker(rank, world, port, n, q):
    import datetime

    import torch.distributed as dist

    from monomers2026_b200.decomposed import TorchTransport
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        lay = SlabLayout(n, world)
        full = _global(lay)
        T = TorchTransport()
        z0, nzl = lay.planes(rank)
        cols, back = _exchange_round(lay, T, [full[:, z0:z0 + nzl].clone()])
        ok = True
        try:
            _check(lay, [rank], cols, back, full)
        except AssertionError:
            ok = False
        g = torch.full((5,), float(rank + 1), dtype=torch.float64)
        T.allreduce_sum([g])
        q.put((rank, ok, g.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n", [(2, 32), (4, 64)])
def test_gloo_ranks_exchange(world, n):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, n, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok, _ in res)
    total = world * (world + 1) / 2
    assert all(g == [total] * 5 for _, _, g in res)


def test_slab_create_refuses_what_it_cannot_decompose():
    """The argument checks of selm_slab_create come before any device work."""
    import ctypes as C

    from monomers2026_b200 import _lib
    from monomers2026_b200.selm import Params

    L = _lib.load()
    h = C.c_void_p()
    cases = [
        (dict(numMeshPtsPerDir=(64, 64, 64), form="fused32"), 2, 2),          # rank outside [0, nranks)
        (dict(numMeshPtsPerDir=(64, 64, 64), form="fused32"), 0, 0),          # no ranks
        (dict(numMeshPtsPerDir=(64, 64, 64), form="plain64"), 0, 2),          # the plain form
        (dict(numMeshPtsPerDir=(64, 64, 64), form="fused32", integrator="quasi_steady"), 0, 2),
        (dict(numMeshPtsPerDir=(64, 64, 64), form="fused64"), 0, 8),          # 64 planes: not 16 per rank
        (dict(numMeshPtsPerDir=(30, 30, 30), form="fused32"), 0, 1),          # no whole 16-plane layers
        (dict(numMeshPtsPerDir=(80, 80, 80), form="fused32"), 0, 1),          # not a compile-time FFT size
    ]
    for kw, rank, nranks in cases:
        p = Params(**kw).to_c()
        assert L.selm_slab_create(C.byref(p), rank, nranks, C.byref(h)) == 1, (kw, rank, nranks)  # SELM_ERR_INVALID
        assert L.selm_last_error()
