"""One instance decomposed over ranks in z slabs: the counterpart of the
reference's MPI path (z slabs with FFTW-MPI transposed layouts,
mpi/SELM_Eulerian_Period.cpp:18-51,348-407; the interpolation summed over
the ranks, mpi/SELM_Lagrangian_LAMMPS.cpp:102).

Each rank holds one slab (``selm_slab_create``): its grid planes, a block of
half-spectrum columns for the z pass, and every monomer.  A step runs the
four stages of the C ABI with two kinds of exchange between them, done by a
``Transport``:

* ``allreduce_sum`` - the interpolation, summed over the ranks;
* ``alltoall`` - the xy spectrum of the slabs' planes to the ranks' columns,
  and back (rank r sends rank s the columns of s from its own planes).

``TorchTransport`` exchanges through ``torch.distributed`` (one process per
GPU: NCCL over NVLink; gloo on CPU tensors, where point-to-point sends
stand in for the all-to-all).  ``LoopbackTransport`` holds every rank's slab
in one process and exchanges by device copies: it runs a decomposed
instance on one GPU, which the tests compare with the whole instance.  The
exchanges are pure data movement; every stage's arithmetic is the
library's own kernels.
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from .selm import Params, Selm, Topology, check


class Transport:
    """Exchanges between the slabs that this process holds (``local``: their
    ranks, in order).  ``allreduce_sum(bufs)``: every buffer (one per local
    slab) becomes the sum over all ranks.  ``alltoall(send, recv)``:
    ``send[i][s]`` goes from local slab i to rank s, where it lands in
    ``recv[k][r]`` (k the local index of rank s, r the sending rank)."""

    nranks: int
    local: list

    def allreduce_sum(self, bufs):
        raise NotImplementedError

    def alltoall(self, send, recv):
        raise NotImplementedError


class LoopbackTransport(Transport):
    """All ranks in this process; exchanges are copies (sums in rank order)."""

    def __init__(self, nranks: int):
        self.nranks = int(nranks)
        self.local = list(range(self.nranks))

    def allreduce_sum(self, bufs):
        total = bufs[0].clone()
        for b in bufs[1:]:
            total += b
        for b in bufs:
            b.copy_(total)

    def alltoall(self, send, recv):
        for r in range(self.nranks):
            for s in range(self.nranks):
                recv[s][r].copy_(send[r][s])


class TorchTransport(Transport):
    """One rank per process through torch.distributed (the default group
    unless ``group`` is given).  NCCL: ``all_reduce`` and ``all_to_all``;
    other backends (gloo): ``all_reduce`` and paired point-to-point sends."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self._dist = dist
        self.group = group
        self.nranks = dist.get_world_size(group)
        self.rank = dist.get_rank(group)
        self.local = [self.rank]
        self.nccl = dist.get_backend(group) == "nccl"

    def allreduce_sum(self, bufs):
        (b,) = bufs
        self._dist.all_reduce(b, op=self._dist.ReduceOp.SUM, group=self.group)

    def alltoall(self, send, recv):
        (snd,), (rcv,) = send, recv
        if self.nccl:
            self._dist.all_to_all(rcv, snd, group=self.group)
            return
        reqs, keep = [], []
        for peer in range(self.nranks):
            if peer == self.rank:
                rcv[peer].copy_(snd[peer])
                continue
            t = snd[peer].contiguous()
            keep.append(t)  # referenced until its send completes
            reqs.append(self._dist.isend(t, peer, group=self.group))
            reqs.append(self._dist.irecv(rcv[peer], peer, group=self.group))
        for q in reqs:
            q.wait()


@dataclasses.dataclass(frozen=True)
class SlabLayout:
    """Planes and columns of each rank for an n^3 grid over ``nranks`` ranks
    (as ``selm_slab_create`` lays them out): rank r holds planes
    [r n/R, (r+1) n/R) and columns [r C, min((r+1) C, ncol)) of the ncol =
    n (n/2+1) half-spectrum columns, C = ceil(ncol / R)."""

    n: int
    nranks: int

    @property
    def nzl(self) -> int:
        return self.n // self.nranks

    @property
    def ncol(self) -> int:
        return self.n * (self.n // 2 + 1)

    def planes(self, r: int) -> tuple[int, int]:
        return r * self.nzl, self.nzl

    def cols(self, r: int) -> tuple[int, int]:
        per = -(-self.ncol // self.nranks)
        c0 = min(self.ncol, r * per)
        return c0, min(self.ncol, c0 + per) - c0


# Exchange buffers are real views of the complex arrays, [..., 2].
# work of rank r: [3][nzl][ncol][2] (its planes); cols of rank r: [3][n][ncl_r][2].

def pack_to_columns(work, lay: SlabLayout) -> list:
    """What a rank sends each rank s on the way to the z pass: its planes of
    rank s's columns, [3][nzl][ncl_s][2]."""
    out = []
    for s in range(lay.nranks):
        c0, ncl = lay.cols(s)
        out.append(work[:, :, c0:c0 + ncl].contiguous())
    return out


def unpack_columns(recv: list, cols, lay: SlabLayout) -> None:
    """recv[s] (rank s's planes of this rank's columns) into cols [3][n][ncl][2]."""
    for s in range(lay.nranks):
        z0, nzl = lay.planes(s)
        cols[:, z0:z0 + nzl].copy_(recv[s])


def pack_to_planes(cols, lay: SlabLayout) -> list:
    """What a rank sends each rank s after the z pass: rank s's planes of its
    own columns, [3][nzl][ncl][2]."""
    out = []
    for s in range(lay.nranks):
        z0, nzl = lay.planes(s)
        out.append(cols[:, z0:z0 + nzl].contiguous())
    return out


def unpack_planes(recv: list, work, lay: SlabLayout) -> None:
    """recv[s] (rank s's columns of this rank's planes) into work [3][nzl][ncol][2]."""
    for s in range(lay.nranks):
        c0, ncl = lay.cols(s)
        work[:, :, c0:c0 + ncl].copy_(recv[s])


def recv_buffers(lay: SlabLayout, rank: int, like) -> tuple[list, list]:
    """Receive buffers of one rank: (to columns, to planes)."""
    import torch

    _, ncl = lay.cols(rank)
    to_cols = [torch.empty((3, lay.nzl, ncl, 2), dtype=like.dtype, device=like.device) for _ in range(lay.nranks)]
    to_planes = [torch.empty((3, lay.nzl, lay.cols(s)[1], 2), dtype=like.dtype, device=like.device)
                 for s in range(lay.nranks)]
    return to_cols, to_planes


class _DeviceArray:
    """A library-owned device array, seen by torch without a copy."""

    def __init__(self, ptr: int, shape: tuple, fp32: bool):
        self.__cuda_array_interface__ = {"shape": tuple(int(v) for v in shape), "typestr": "<f4" if fp32 else "<f8",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def _device_tensor(ptr: int, shape: tuple, fp32: bool):
    import torch

    return torch.as_tensor(_DeviceArray(ptr, shape, fp32), device="cuda")


class Decomposed:
    """One instance over ``transport.nranks`` ranks in z slabs; this process
    steps the slabs of ``transport.local`` (all of them with a
    ``LoopbackTransport``).  Every rank is given the same monomers and
    topology and keeps all of them.  The slabs run on one torch stream of
    their own, and every exchange is issued on it, so that the copies and the
    collectives are ordered with the stages."""

    def __init__(self, params: Params, x: np.ndarray, mass: np.ndarray, v: np.ndarray | None = None,
                 topology: Topology | None = None, transport: Transport | None = None):
        import torch

        if params.form not in ("fused32", "fused64"):
            raise ValueError("a decomposed instance runs the fused forms")
        self.transport = transport if transport is not None else LoopbackTransport(1)
        self.layout = SlabLayout(int(params.numMeshPtsPerDir[0]), self.transport.nranks)
        self.fp32 = params.form == "fused32"
        self.slabs = [Selm(params, x, mass, v=v, topology=topology, slab=(r, self.transport.nranks))
                      for r in self.transport.local]
        self.M = self.slabs[0].M
        self._stream = torch.cuda.Stream()
        for s in self.slabs:
            s.set_stream(self._stream.cuda_stream)
        self._bufs = []

    def initial(self) -> None:
        import torch

        with torch.cuda.stream(self._stream):
            self._initial()

    def _initial(self) -> None:
        for s in self.slabs:
            s.initial()
        L = _lib.load()
        lay = self.layout
        self._bufs = []
        for r, s in zip(self.transport.local, self.slabs):
            g, w, c = C.c_void_p(), C.c_void_p(), C.c_void_p()
            sizes = (C.c_longlong * 3)()
            check(L.selm_slab_buffers(s._h, C.byref(g), C.byref(w), C.byref(c), sizes))
            ncl = lay.cols(r)[1]
            gather = _device_tensor(g.value, (3 * self.M,), self.fp32) if self.M else None
            work = _device_tensor(w.value, (3, lay.nzl, lay.ncol, 2), self.fp32)
            cols = _device_tensor(c.value, (3, lay.n, ncl, 2), self.fp32)
            self._bufs.append((gather, work, cols) + recv_buffers(lay, r, work))

    def step(self, nsteps: int = 1) -> None:
        import torch

        with torch.cuda.stream(self._stream):
            self._step(nsteps)

    def _step(self, nsteps: int) -> None:
        L = _lib.load()
        lay, T = self.layout, self.transport
        for _ in range(int(nsteps)):
            for s in self.slabs:
                check(L.selm_slab_gather(s._h))
            if self.M:
                T.allreduce_sum([b[0] for b in self._bufs])
            for s in self.slabs:
                check(L.selm_slab_advance(s._h))
            T.alltoall([pack_to_columns(b[1], lay) for b in self._bufs], [b[3] for b in self._bufs])
            for b in self._bufs:
                unpack_columns(b[3], b[2], lay)
            for s in self.slabs:
                check(L.selm_slab_solve(s._h))
            T.alltoall([pack_to_planes(b[2], lay) for b in self._bufs], [b[4] for b in self._bufs])
            for b in self._bufs:
                unpack_planes(b[4], b[1], lay)
            for s in self.slabs:
                check(L.selm_slab_finish(s._h))

    run = step

    def particles(self):
        """x, v, f (the same on every rank)."""
        return self.slabs[0].particles()

    def velocity(self) -> dict:
        """The fluid velocity of this process's slabs: {rank: [3][nzl][n][n]}."""
        L = _lib.load()
        n, nzl = self.layout.n, self.layout.nzl
        out = {}
        for r, s in zip(self.transport.local, self.slabs):
            a = np.zeros((3, nzl, n, n))
            check(L.selm_slab_velocity(s._h, a.ctypes.data_as(C.POINTER(C.c_double))))
            out[r] = a
        return out

    def status(self) -> int:
        w = 0
        for s in self.slabs:
            w |= s.status()
        return w

    def final(self) -> None:
        for s in self.slabs:
            s.final()
