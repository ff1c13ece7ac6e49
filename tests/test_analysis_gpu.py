"""On-device analysis (selm_analysis_*) against the oracle on the same
trajectory: the positions and velocities read back at every sample.

MSD sums: 1e-12 relative (the float32 frames and the FP64 fold are the same
numbers; only the summation order differs).  The same sums also come out of
the reference's MSD.py loop run on the DCD file written at the same samples.
S(q): 1e-9 relative plus 1e-10 absolute (sincospi vs cos/sin of the phase).
K_d: 1e-12 relative.  Repeated runs, and runs inside a batch, are bitwise
equal."""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from oracle import analysis as oa

pytestmark = pytest.mark.gpu

NLAG, STRIDE, EVERY, SAMPLES = 6, 2, 5, 30


def _sim(form, seed=11, n=32):
    from monomers2026_b200.serving import _make
    from monomers2026_b200.workloads import replica
    return _make(replica(n, 10, 20, 1.0, seed, form=form))


def _run(s, a, dcd=None, lib=None):
    xs, vs = [], []
    for k in range(SAMPLES):
        if k:
            s.run(EVERY)
        a.sample()
        x, v, _ = s.particles()
        xs.append(x)
        vs.append(v)
        if dcd is not None:
            assert lib.selm_dcd_write_sim(dcd, s._h) == 0
    return np.array(xs), np.array(vs)


@pytest.mark.parametrize("form", ["fused32", "fused64", "plain64"])
def test_analysis_matches_oracle(form):
    from monomers2026_b200 import _lib
    from monomers2026_b200.analysis import Analysis, wavevectors
    from monomers2026_b200.dcd import read_dcd
    L_ = _lib.load()
    s = _sim(form)
    q = wavevectors(2)
    a = Analysis(s, nlag=NLAG, lag_stride=STRIDE, qvec=q)
    with tempfile.TemporaryDirectory() as tmp:
        h = C.c_void_p()
        assert L_.selm_dcd_open_sim(os.path.join(tmp, "t.dcd").encode(), s._h, EVERY, C.byref(h)) == 0
        xs, vs = _run(s, a, h, L_)
        assert L_.selm_dcd_close(h) == 0
        traj = read_dcd(os.path.join(tmp, "t.dcd"))
    box = s.params.box_hi - s.params.box_lo
    sums, pairs = a.msd_sums()
    osum, opairs = oa.msd_sums(xs, box, NLAG, STRIDE)
    assert np.array_equal(pairs, opairs)
    assert np.allclose(sums, osum, rtol=1e-12, atol=0)
    assert np.all(sums > 0)
    # MSD.py on the DCD written at the same samples
    lit, lsum = oa.msd_literal(traj["xyz"], traj["cells"][0][0], dotnum=NLAG + 1, mult=STRIDE, start_fraction=0.0)
    assert np.allclose(lsum[1:], sums, rtol=1e-12, atol=0)
    lag, msd = a.msd()
    assert np.allclose(msd, lit[1:], rtol=1e-12)
    # S(q) and K_d
    sq, sq_err, k = a.structure()
    assert k == SAMPLES
    osq = np.array([oa.structure_factor(x, box, q) for x in xs])
    assert np.allclose(sq, osq.mean(axis=0), rtol=1e-9, atol=1e-10)
    ke, ke_err, k = a.kinetic()
    oke = np.array([oa.kinetic(v, np.ones(len(v))) for v in vs])
    assert np.allclose(ke, oke.mean(axis=0), rtol=1e-12)
    assert np.allclose(ke_err, oke.std(axis=0) / np.sqrt(SAMPLES - 1), rtol=1e-6)
    assert a.device_bytes() > 0
    a.close()
    s.final()


def test_analysis_repeats_bitwise_and_in_batch():
    from monomers2026_b200.analysis import Analysis, wavevectors
    from monomers2026_b200.selm import Batch
    q = wavevectors(1)

    def alone(seed):
        s = _sim("fused32", seed)
        a = Analysis(s, NLAG, STRIDE, q)
        for k in range(SAMPLES):
            if k:
                s.run(EVERY)
            a.sample()
        out = (a.msd_sums()[0], a.structure()[0], a.kinetic()[0])
        a.close()
        s.final()
        return out

    r1, r2 = alone(11), alone(11)
    for u, w in zip(r1, r2):
        assert np.array_equal(u, w)
    sims = [_sim("fused32", 11), _sim("fused32", 12, n=48)]
    ans = [Analysis(s, NLAG, STRIDE, q) for s in sims]
    b = Batch()
    for s in sims:
        b.add(s)
    for k in range(SAMPLES):
        if k:
            b.run(EVERY)
        for a in ans:
            a.sample()
    rb = (ans[0].msd_sums()[0], ans[0].structure()[0], ans[0].kinetic()[0])
    for u, w in zip(r1, rb):
        assert np.array_equal(u, w)
    b.final()
    rb2 = (ans[1].msd_sums()[0], ans[1].structure()[0], ans[1].kinetic()[0])
    for a in ans:
        a.close()
    for s in sims:
        s.final()
    s = _sim("fused32", 12, n=48)
    a = Analysis(s, NLAG, STRIDE, q)
    for k in range(SAMPLES):
        if k:
            s.run(EVERY)
        a.sample()
    for u, w in zip((a.msd_sums()[0], a.structure()[0], a.kinetic()[0]), rb2):
        assert np.array_equal(u, w)
    a.close()
    s.final()


def test_analysis_outlives_its_simulation_safely():
    from monomers2026_b200.analysis import Analysis
    s = _sim("fused32")
    a = Analysis(s, 2, 1)
    a.sample()
    s.final()
    with pytest.raises(Exception):
        a.sample()
    with pytest.raises(Exception):
        a.msd_sums()
    a.close()


def test_reset_and_lags_without_pairs():
    from monomers2026_b200.analysis import Analysis
    s = _sim("fused32")
    a = Analysis(s, 4, 3)
    for _ in range(5):
        a.sample()
        s.run(2)
    sums, pairs = a.msd_sums()
    assert list(pairs) == [2 * s.M, 0, 0, 0]
    assert sums[0].sum() > 0 and np.all(sums[1:] == 0)
    lag, msd = a.msd()
    assert np.isfinite(msd[0]) and np.all(np.isnan(msd[1:]))
    a.reset()
    sums, pairs = a.msd_sums()
    assert np.all(sums == 0) and np.all(pairs == 0)
    a.close()
    s.final()


def test_analysis_without_monomers():
    """A fluid-only simulation: sampling counts, and every sum stays zero."""
    from monomers2026_b200 import workloads as W
    from monomers2026_b200.analysis import Analysis, wavevectors
    from monomers2026_b200.selm import Selm
    wl = W.config(1, kT=1.0, grid=16, form="fused32")
    s = Selm(wl.params, wl.x[:0].copy(), wl.mass[:0].copy())
    s.initial()
    a = Analysis(s, 3, 1, wavevectors(1))
    for _ in range(4):
        s.run(1)
        a.sample()
    sums, pairs = a.msd_sums()
    assert np.all(sums == 0) and np.all(pairs == 0)
    sq, _, k = a.structure()
    assert k == 4 and np.all(sq == 0)
    kd, _, k = a.kinetic()
    assert k == 4 and np.all(kd == 0)
    assert s.status() == 0
    a.close()
    s.final()
