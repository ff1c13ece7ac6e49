"""Batched stepping (selm_batch_*) on a B200.

A member of a batch runs its own captured step graph as a child of the
batch's graph, with its own buffers and Philox counters, so its state after
any number of batch steps must equal, bit for bit, the state of the same
simulation stepped alone; members joining and leaving between steps
(continuous batching) must not change that.
"""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Batch, Selm

pytestmark = pytest.mark.gpu


def _sim(wl):
    s = Selm(wl.params, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    s.initial()
    return s


def _state(s):
    x, v, f = s.particles()
    return x, v, f, s.get_field(0)


def _same(a, b):
    return all(np.array_equal(p, q) for p, q in zip(a, b))


@pytest.mark.parametrize("form", ["fused32", "fused64"])
def test_batch_equals_alone(form):
    specs = [(16, 2, 12, 1.0, 11), (24, 3, 20, 0.7, 12), (32, 1, 50, 1.5, 13), (16, 1, 8, 0.0, 14)]
    alone, inb = [], []
    for n, nc, ln, kT, seed in specs:
        alone.append(_sim(W.replica(n, nc, ln, kT, seed, form=form)))
        inb.append(_sim(W.replica(n, nc, ln, kT, seed, form=form)))
    for s in alone:
        s.run(7)
    b = Batch()
    for s in inb:
        b.add(s)
    assert len(b) == len(specs)
    b.run(7)
    for s, t in zip(alone, inb):
        assert _same(_state(s), _state(t))
        assert t.nstep == 7 and t.status() == 0
    b.final()


def test_continuous_batching_join_and_leave():
    mk = lambda n, nc, kT, seed: _sim(W.replica(n, nc, 10, kT, seed))
    specs = {"a": (16, 2, 1.0, 21), "b": (24, 2, 0.5, 22), "c": (32, 3, 2.0, 23)}
    ref = {k: mk(*v) for k, v in specs.items()}
    sim = {k: mk(*v) for k, v in specs.items()}
    b = Batch()
    b.add(sim["a"])
    b.add(sim["b"])
    b.run(5)
    b.add(sim["c"])  # joins at step 5 of a and b
    b.run(3)
    b.remove(sim["a"])  # leaves after 8 steps
    b.run(4)
    ref["a"].run(8)
    ref["b"].run(12)
    ref["c"].run(7)
    for k in "abc":
        assert _same(_state(ref[k]), _state(sim[k])), k
    # a left the batch: it steps alone again, on its own stream
    sim["a"].run(2)
    ref["a"].run(2)
    assert _same(_state(ref["a"]), _state(sim["a"]))
    b.final()


def test_batch_member_rules():
    s = _sim(W.replica(16, 1, 10, 1.0, 31))
    b = Batch()
    b.add(s)
    with pytest.raises(Exception):
        s.run(1)  # members step through their batch
    with pytest.raises(Exception):
        b.add(s)  # once
    p = _sim(W.replica(16, 1, 10, 1.0, 32, form="plain64"))
    with pytest.raises(Exception):
        b.add(p)  # the plain form has no captured step
    b.final()
    s.run(1)  # after the batch is gone the simulation steps alone


def test_device_bytes_grow_with_the_grid():
    small = _sim(W.replica(16, 1, 10, 1.0, 41))
    large = _sim(W.replica(48, 1, 10, 1.0, 42))
    bs, bl = small.device_bytes(), large.device_bytes()
    assert 0 < bs < bl
    # FP32 fused state: u, the spread grid (3N floats each), work and u_hat (3 N2 complex each)
    N = 48 ** 3
    N2 = 25 * 48 * 48
    assert bl > 4 * 3 * N * 2 + 8 * 3 * N2 * 2
