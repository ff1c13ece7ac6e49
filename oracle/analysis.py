"""TEST INFRASTRUCTURE ONLY: CPU restatement of the reference's trajectory
analysis, the checker of the on-device analysis (selm_analysis_*).

Only tests/ import this module; the product never does.

``msd_literal`` follows data/src/Diffusion Coefficient/MSD.py:14-91 loop for
loop (NumPy 1.26 promotion: frames are float32, the difference of two frame
values is float32, the fold by 2X, the square and the sums are float64).
``msd_sums`` is the same arithmetic vectorised; ``structure_factor`` and
``kinetic`` restate the S(q) and equipartition sums the device accumulates.
"""
from __future__ import annotations

import numpy as np


def _fold(dd: np.ndarray, half: float) -> np.ndarray:
    """MSD.py:59-66: one shift by the box when |d| reaches half of it."""
    d = dd.astype(np.float64)
    return np.where(d >= half, d - 2.0 * half, np.where(d <= -half, d + 2.0 * half, d))


def msd_literal(frames: np.ndarray, box: float, dotnum: int, mult: int, start_fraction: float = 0.2):
    """MSD.py:14-91 on frames [F][M][3] (float32, as read from a DCD):
    frames from int(F * start_fraction) on (MSD.py:30: numframes / 5), lags
    dot*mult for dot = 1 .. dotnum-1.  Returns (MSD[0:dotnum], per-direction
    sums [dotnum][3]); MSD[0] = 0."""
    fr = np.asarray(frames, dtype=np.float32)
    F, M, _ = fr.shape
    start = int(F * start_fraction)
    fr = fr[start:]
    Fn = len(fr)
    X = float(np.float32(box)) / 2
    out = [0.0] * dotnum
    sums = np.zeros((dotnum, 3))
    for dot in range(1, dotnum):
        lag = dot * mult
        acc = [0.0, 0.0, 0.0]
        Fd = Fn - lag
        for idx in range(M):
            for n in range(0, Fd):
                for d in range(3):
                    t = float(np.float32(fr[n + lag, idx, d] - fr[n, idx, d]))
                    if t >= X:
                        acc[d] += (t - 2 * X) ** 2
                    if t <= -X:
                        acc[d] += (t + 2 * X) ** 2
                    if -X < t < X:
                        acc[d] += t ** 2
        sums[dot] = acc
        out[dot] = (acc[0] + acc[1] + acc[2]) / (Fd * M) if Fd > 0 else float("nan")
    return np.array(out), sums


def msd_sums(frames: np.ndarray, box: float, nlag: int, stride: int):
    """Per-direction sums [nlag][3] and pair counts [nlag] (pairs x monomers)
    over all frame pairs (n, n + l*stride), l = 1..nlag, of frames [F][M][3]
    (rounded to float32 first)."""
    fr = np.asarray(frames, dtype=np.float64).astype(np.float32)
    F, M, _ = fr.shape
    half = float(np.float32(box)) / 2
    sums = np.zeros((nlag, 3))
    pairs = np.zeros(nlag, dtype=np.int64)
    for l in range(1, nlag + 1):
        lag = l * stride
        if lag >= F:
            continue
        dd = fr[lag:] - fr[:F - lag]  # float32 differences
        t = _fold(dd, half)
        sums[l - 1] = (t * t).sum(axis=(0, 1))
        pairs[l - 1] = (F - lag) * M
    return sums, pairs


def structure_factor(x: np.ndarray, box: float, qvec: np.ndarray) -> np.ndarray:
    """|sum_j exp(i 2 pi n.x_j / L)|^2 / M for each integer triple n."""
    x = np.asarray(x, dtype=np.float64)
    ph = 2.0 * np.pi * (x @ np.asarray(qvec, dtype=np.float64).T) / box  # [M][nq]
    re = np.cos(ph).sum(axis=0)
    im = np.sin(ph).sum(axis=0)
    return (re * re + im * im) / len(x)


def kinetic(v: np.ndarray, m: np.ndarray) -> np.ndarray:
    """K_d = sum_j m_j v_jd^2 per direction."""
    v = np.asarray(v, dtype=np.float64)
    return (np.asarray(m, dtype=np.float64)[:, None] * v * v).sum(axis=0)
