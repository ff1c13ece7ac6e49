"""Batched stepping (selm_batch_*) on a B200.

A member of a batch runs its own captured step graph as a child of its
group's graph, with its own buffers and Philox counters, so its state after
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


def test_read_back_around_joining_and_leaving():
    """Read back right after stepping alone (the read-back that overlaps the
    rest of that step), then after batch steps (on the batch's stream), then
    after leaving: every read-back equals that of the same simulation
    stepped alone throughout."""
    mk = lambda: _sim(W.replica(24, 3, 20, 1.0, 31))
    ref, s = mk(), mk()
    b = Batch()
    for alone_steps, batch_steps in ((2, 3), (1, 2)):
        s.run(alone_steps)
        ref.run(alone_steps)
        assert _same(s.particles(), ref.particles())
        b.add(s)
        b.run(batch_steps)
        ref.run(batch_steps)
        assert _same(s.particles(), ref.particles())
        b.remove(s)
        assert _same(s.particles(), ref.particles())
    assert _same(_state(s), _state(ref))
    b.final()


def test_groups_shared_by_several_members():
    """More members than groups (eight): groups hold two members each; a
    member leaving a shared group and members joining at odd steps (other
    position parities) rebuild only their groups, and every member still
    equals its solo run bit for bit."""
    mk = lambda seed: _sim(W.replica(16 if seed % 2 else 24, 1 + seed % 3, 10, 1.0, seed))
    seeds = list(range(60, 73))  # 13 members
    ref = {k: mk(k) for k in seeds}
    sim = {k: mk(k) for k in seeds}
    b = Batch()
    for k in seeds[:10]:
        b.add(sim[k])
    b.run(3)
    b.remove(sim[seeds[8]])  # shares a group with seeds[0]
    b.add(sim[seeds[10]])
    b.run(2)
    b.add(sim[seeds[11]])
    b.add(sim[seeds[12]])
    b.run(4)
    assert len(b) == 12
    done = {k: 9 for k in seeds[:10]}
    done[seeds[8]] = 3
    done[seeds[10]] = 6
    done[seeds[11]] = done[seeds[12]] = 4
    for k in seeds:
        ref[k].run(done[k])
        assert sim[k].nstep == done[k]
        assert _same(_state(ref[k]), _state(sim[k])), k
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


def test_server_results_same_alone_and_in_mix():
    from monomers2026_b200.serving import Server, estimate_device_bytes, serving_jobs

    jobs = serving_jobs(6, rate=2000.0, grids=(16, 24, 32), weights=(1, 1, 1), m_range=(20, 200),
                        steps_range=(5, 20), seed=77)
    # a budget of about three jobs: later arrivals wait in the queue for memory
    per = [estimate_device_bytes(j.workload.params, len(j.workload.mass)) for j in jobs]
    srv = Server(budget_bytes=int(3.2 * max(per)))
    out = srv.run(jobs)
    srv.final()
    assert out["jobs"] == 6 and out["status_nonzero"] == 0
    assert out["max_batch"] >= 2  # jobs overlapped on the device
    for j in jobs:
        s = _sim(j.workload)
        s.run(j.nsteps)
        x, v, _ = s.particles()
        assert np.array_equal(x, j.x) and np.array_equal(v, j.v), j.jid
        s.final()


def test_estimate_covers_device_bytes():
    from monomers2026_b200.serving import estimate_device_bytes

    for n, M in ((16, 20), (32, 500), (64, 3000)):
        wl = W.replica(n, 1, M, 1.0, 50 + n)
        s = _sim(wl)
        est = estimate_device_bytes(wl.params, M)
        assert s.device_bytes() <= est < 3 * s.device_bytes() + (8 << 20), (n, M, s.device_bytes(), est)
        s.final()


def test_jobs_poll_and_retire_match_alone():
    """Jobs with step budgets (selm_batch_add_job): each leaves the step
    graphs when its budget is spent, selm_batch_poll reports it once its last
    step has finished, and selm_batch_retire reads it back on its own stream;
    the states equal the same simulations stepped alone, bit for bit.  A job
    whose budget is not spent cannot be retired."""
    wls = [W.replica(16, 1, 40, 1.0, 801), W.replica(24, 1, 120, 0.7, 802), W.replica(16, 2, 30, 1.5, 803)]
    budgets = [3, 7, 5]
    b = Batch()
    sims = [_sim(w) for w in wls]
    for s, n in zip(sims, budgets):
        b.add_job(s, n)
    with pytest.raises(RuntimeError):
        b.retire(sims[0])
    got = {}
    for _ in range(12):
        b.run(1)
        b.synchronize()
        for s in b.poll():
            got[sims.index(s)] = b.retire(s)
    assert sorted(got) == [0, 1, 2] and len(b) == 0
    for i, (w, n) in enumerate(zip(wls, budgets)):
        alone = _sim(w)
        alone.run(n)
        x, v, f = alone.particles()
        assert np.array_equal(x, got[i][0]) and np.array_equal(v, got[i][1]) and np.array_equal(f, got[i][2]), i
        alone.final()
        assert sims[i].status() == 0
        sims[i].final()
    b.final()
