"""On-device analysis of a running simulation (selm_analysis_* of the C ABI).

The reference analyses its runs after the fact: LAMMPS dumps a DCD
trajectory, ``MSD.py`` computes the mean square displacement of the monomers
over frame lags (data/src/Diffusion Coefficient/MSD.py:14-91) and a straight
line fitted to MSD(t) gives the diffusion coefficient (get_K.py,
compare_period_2MSD/comapre_MSD.py:linear_fit).  ``Analysis`` accumulates the
same MSD sums on the device while the simulation runs (no trajectory is
written or read back), together with the static structure factor and the
kinetic energy per direction (equipartition); ``fit_line`` and
``diffusion_coefficient`` are the fits.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def wavevectors(nmax: int) -> np.ndarray:
    """Integer triples n with 0 < |n|^2 <= nmax^2, one of each +-n pair
    (S(q) = S(-q)), sorted by |n|."""
    r = np.arange(-nmax, nmax + 1)
    g = np.stack(np.meshgrid(r, r, r, indexing="ij"), axis=-1).reshape(-1, 3)
    n2 = (g * g).sum(axis=1)
    keep = (n2 > 0) & (n2 <= nmax * nmax)
    g = g[keep]
    # one of +-n: first non-zero component positive
    first = np.where(g[:, 0] != 0, g[:, 0], np.where(g[:, 1] != 0, g[:, 1], g[:, 2]))
    g = g[first > 0]
    return g[np.argsort((g * g).sum(axis=1), kind="stable")].astype(np.int32)


class Analysis:
    """MSD over ``nlag`` lags of ``lag_stride`` samples, S(q) at ``qvec``
    (integer triples, q = 2 pi n / L) and K_d, accumulated at every
    ``sample()`` on the simulation's stream."""

    def __init__(self, sim, nlag: int = 40, lag_stride: int = 1, qvec=None):
        self._L = _lib.load()
        self.sim = sim  # keeps the simulation alive while the analysis is used
        q = np.zeros((0, 3), np.int32) if qvec is None else np.ascontiguousarray(qvec, dtype=np.int32).reshape(-1, 3)
        self.qvec = q
        self.nlag, self.lag_stride = int(nlag), int(lag_stride)
        h = C.c_void_p()
        check(self._L.selm_analysis_create(sim._h, self.nlag, self.lag_stride, len(q),
                                           q.ctypes.data_as(C.POINTER(C.c_int)) if len(q) else None, C.byref(h)))
        self._h = h

    def sample(self) -> None:
        check(self._L.selm_analysis_sample(self._h))

    def msd_sums(self):
        """(sums [nlag][3], pairs [nlag]): per-direction sums of squared
        folded displacements and (frame pairs x monomers) per lag."""
        s = np.zeros((self.nlag, 3))
        p = np.zeros(self.nlag, dtype=np.int64)
        check(self._L.selm_analysis_msd(self._h, _dp(s), p.ctypes.data_as(C.POINTER(C.c_longlong))))
        return s, p

    def msd(self):
        """(lag in samples [nlag], MSD [nlag]); NaN where no pair was seen."""
        s, p = self.msd_sums()
        with np.errstate(invalid="ignore", divide="ignore"):
            m = np.where(p > 0, s.sum(axis=1) / np.maximum(p, 1), np.nan)
        return np.arange(1, self.nlag + 1) * self.lag_stride, m

    def msd_curve(self, dt: float, sample_every: int, tau: float = 1.0):
        """MSD.py's output: time = lag x dt x steps between samples / tau,
        with the point (0, 0) first (MSD.py:53-56)."""
        lag, m = self.msd()
        return np.concatenate([[0.0], lag * dt * sample_every / tau]), np.concatenate([[0.0], m])

    def _moments(self, fn, n):
        s, s2 = np.zeros(n), np.zeros(n)
        k = C.c_longlong()
        check(fn(self._h, _dp(s), _dp(s2), C.byref(k)))
        k = int(k.value)
        if k == 0:
            return np.full(n, np.nan), np.full(n, np.nan), 0
        mean = s / k
        var = np.maximum(s2 / k - mean * mean, 0.0)
        return mean, np.sqrt(var / max(k - 1, 1)), k

    def structure(self):
        """(mean S(q), standard error, samples); samples are correlated in
        time, so the error is a lower bound unless they are spaced out."""
        return self._moments(self._L.selm_analysis_structure, len(self.qvec))

    def kinetic(self):
        """(mean K_d, standard error, samples) per direction; the
        equipartition value of K_d / M is kT."""
        return self._moments(self._L.selm_analysis_kinetic, 3)

    def reset(self) -> None:
        check(self._L.selm_analysis_reset(self._h))

    def device_bytes(self) -> int:
        n = C.c_ulonglong()
        check(self._L.selm_analysis_device_bytes(self._h, C.byref(n)))
        return int(n.value)

    def close(self) -> None:
        if self._h:
            self._L.selm_analysis_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fit_line(t, y, tmin: float | None = None, tmax: float | None = None):
    """Least-squares straight line y = k t + b over tmin <= t <= tmax (the
    reference's linear_fit / curve_fit of a line).  Returns (k, b)."""
    t = np.asarray(t, dtype=float)
    y = np.asarray(y, dtype=float)
    m = np.isfinite(y)
    if tmin is not None:
        m &= t >= tmin
    if tmax is not None:
        m &= t <= tmax
    k, b = np.polyfit(t[m], y[m], 1)
    return float(k), float(b)


def diffusion_coefficient(t, msd, tmin: float | None = None, tmax: float | None = None) -> float:
    """D = slope / 6 of MSD(t) in three dimensions (Einstein relation)."""
    return fit_line(t, msd, tmin, tmax)[0] / 6.0
