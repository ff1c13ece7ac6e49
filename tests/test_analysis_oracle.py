"""The analysis oracle (CPU) against the reference's MSD.py semantics, and
the streaming scheme of the device analysis restated on the CPU.

Pin: the reference's recorded trajectory of its 1base case
(data/cases/SELM/DIffusion Coefficient/1base.dcd) analysed as MSD.py does
(start at frame F/5, lags 5, 10, ... 200 frames) against the reference's own
MSD curve (data/cases/SELM/compare_period_2MSD/1base.txt).  That curve came
from another run of the same case, so agreement is statistical (every lag
within 6%), not bitwise; the arithmetic itself is pinned by the literal
restatement of MSD.py's loops."""
import os

import numpy as np
import pytest

from oracle import analysis as oa
from monomers2026_b200.analysis import fit_line, wavevectors

REF = os.path.join(os.environ.get("SELM_REFERENCE_ROOT", "/root/reference"), "data/cases/SELM")


def _traj(rng, F, M, L):
    """Wrapped random walk with some steps of exactly +-L/2 and near it."""
    x = np.zeros((F, M, 3))
    x[0] = rng.uniform(-L / 2, L / 2, (M, 3))
    for n in range(1, F):
        step = rng.normal(0, 0.15 * L, (M, 3))
        x[n] = x[n - 1] + step
        x[n] = (x[n] + L / 2) % L - L / 2
    x[3, 0, 0] = x[2, 0, 0] + L / 2 if x[2, 0, 0] < 0 else x[2, 0, 0] - L / 2  # exactly half the box
    return x


def test_literal_and_vectorised_msd_agree():
    rng = np.random.default_rng(7)
    L = 6.0
    fr = _traj(rng, 40, 5, L).astype(np.float32)
    lit, lsum = oa.msd_literal(fr, L, dotnum=8, mult=2, start_fraction=0.0)
    s, p = oa.msd_sums(fr, L, nlag=7, stride=2)
    assert np.allclose(lsum[1:], s, rtol=1e-13, atol=0)
    assert np.allclose(lit[1:], s.sum(axis=1) / p, rtol=1e-13)
    assert np.array_equal(p, (40 - 2 * np.arange(1, 8)) * 5)


def test_fold_at_half_box():
    L = 6.0
    fr = np.zeros((2, 4, 3), np.float32)
    fr[1, :, 0] = [3.0, -3.0, 2.9999998, -2.9999998]  # d >= X and d <= -X fold, just inside does not
    s, _ = oa.msd_sums(fr, L, 1, 1)
    d = np.array([3.0 - 6.0, -3.0 + 6.0, np.float32(2.9999998), -np.float32(2.9999998)], dtype=np.float64)
    assert s[0, 0] == pytest.approx((d * d).sum(), rel=1e-15)


def _ring(frames, L, nlag, stride):
    """The device scheme on the CPU: a ring of nlag*stride + 1 float32 frames;
    each new frame adds its pairs with the frames l*stride before it."""
    R = nlag * stride + 1
    M = frames.shape[1]
    ring = np.zeros((R, M, 3), np.float32)
    sums = np.zeros((nlag, 3))
    half = float(np.float32(L)) / 2
    for f, x in enumerate(frames):
        slot = f % R
        xn = x.astype(np.float32)
        nvalid = min(f // stride, nlag)
        for l in range(nvalid):
            old = (slot - (l + 1) * stride + R) % R
            t = oa._fold(xn - ring[old], half)
            sums[l] += (t * t).sum(axis=0)
        ring[slot] = xn
    pairs = np.array([max(0, len(frames) - (l + 1) * stride) * M for l in range(nlag)])
    return sums, pairs


@pytest.mark.parametrize("nlag,stride,F", [(5, 1, 12), (4, 3, 30), (6, 2, 9)])
def test_streaming_ring_equals_all_pairs(nlag, stride, F):
    rng = np.random.default_rng(nlag * 100 + stride)
    L = 8.0
    fr = _traj(rng, F, 7, L)
    s1, p1 = _ring(fr, L, nlag, stride)
    s2, p2 = oa.msd_sums(fr, L, nlag, stride)
    assert np.array_equal(p1, p2)
    assert np.allclose(s1, s2, rtol=1e-13, atol=0)


@pytest.mark.skipif(not os.path.isdir(REF), reason="reference tree not present")
def test_msd_of_reference_trajectory_matches_reference_curve():
    from monomers2026_b200.dcd import read_dcd
    d = read_dcd(os.path.join(REF, "DIffusion Coefficient", "1base.dcd"))
    ref = np.loadtxt(os.path.join(REF, "compare_period_2MSD", "1base.txt"))
    fr = d["xyz"]
    L = d["cells"][0][0]
    start = int(len(fr) / 5)
    s, p = oa.msd_sums(fr[start:], L, nlag=40, stride=5)
    msd = s.sum(axis=1) / p
    t = np.arange(1, 41) * 5 * d["dt"] * d["nsavc"]
    assert np.allclose(t, ref[1:, 0])
    assert np.all(np.abs(msd / ref[1:, 1] - 1) < 0.06)
    # the literal loop on a slice agrees with the vectorised sums
    lit, lsum = oa.msd_literal(fr[start:start + 60], L, dotnum=4, mult=5, start_fraction=0.0)
    s2, _ = oa.msd_sums(fr[start:start + 60], L, nlag=3, stride=5)
    assert np.allclose(lsum[1:], s2, rtol=1e-13)
    # diffusion coefficients of the two curves (slope / 6 over the linear range)
    k_ours, _ = fit_line(t, msd, 500, 4000)
    k_ref, _ = fit_line(ref[1:, 0], ref[1:, 1], 500, 4000)
    assert abs(k_ours / k_ref - 1) < 0.1


def test_structure_factor_of_a_lattice():
    L, n = 4.0, 4
    g = (np.stack(np.meshgrid(*[np.arange(n)] * 3, indexing="ij"), -1).reshape(-1, 3) + 0.5) * (L / n) - L / 2
    q = np.array([[n, 0, 0], [0, 0, n], [1, 0, 0], [1, 1, 0]], np.int32)
    s = oa.structure_factor(g, L, q)
    assert np.allclose(s[:2], len(g)) and np.allclose(s[2:], 0, atol=1e-20 * len(g) + 1e-12)


def test_wavevectors_half_space():
    q = wavevectors(2)
    n2 = (q * q).sum(axis=1)
    assert np.all(np.diff(n2) >= 0) and n2.min() == 1 and n2.max() == 4
    keys = {tuple(v) for v in q}
    assert not any(tuple(-v) in keys for v in q)
    full = [(i, j, k) for i in range(-2, 3) for j in range(-2, 3) for k in range(-2, 3) if 0 < i * i + j * j + k * k <= 4]
    assert 2 * len(q) == len(full)


def test_fit_line():
    t = np.linspace(0, 10, 11)
    assert fit_line(t, 3 * t + 1) == pytest.approx((3.0, 1.0))
    assert fit_line(t, np.where(t > 5, 2 * t, 0 * t), tmin=6) == pytest.approx((2.0, 0.0), abs=1e-12)
