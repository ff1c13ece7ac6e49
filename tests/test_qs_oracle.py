"""The quasi-steady (overdamped) form on the CPU oracle: physics checks.

The form is this project's own (the reference integrates the inertial
scheme only), so it has no reference parity; these tests pin the oracle
restatement with analytic and statistical properties instead:
* the self-mobility of one Peskin 4-point particle in periodic boxes of
  several sizes follows Hasimoto's finite-box correction
  mu(L) = (1 - 2.837297 a/L + 4.19 (a/L)^3 - 27.4 (a/L)^6) / (6 pi mu a)
  with one hydrodynamic radius a (about 1.26 dx for this kernel);
* the velocity is linear in the forces and its grid mean is zero;
* fluctuation-dissipation: over many steps' noise, Var(v) dt / (2 kT)
  equals the deterministic self-mobility (4 sigma of the sample variance);
* the whole step moves x by dt Gamma u(x^n) and ends with F(x^{n+1}).
"""
import numpy as np
import pytest
from scipy.optimize import brentq


def _mobility(O, n, pos, axis=0, mu=1.0):
    x = np.array([pos], dtype=float)
    F = np.zeros((1, 3))
    F[0, axis] = 1.0
    u = O.qs_velocity((n, n, n), 0.0, 1.0, x, F, mu)
    return O.interp(u, 0.0, 1.0, x)[0, axis]


def _hasimoto_radius(m, L, mu=1.0):
    f = lambda a: (1 - 2.837297 * a / L + 4.19 * (a / L) ** 3 - 27.4 * (a / L) ** 6) / (6 * np.pi * mu * a) - m
    return brentq(f, 0.3, 4.0)


def test_qs_mobility_follows_hasimoto(oracle):
    radii = []
    for n in (16, 32):
        m = _mobility(oracle, n, (n / 2 + 0.3, n / 2 + 0.7, n / 2 + 0.1))
        radii.append(_hasimoto_radius(m, n))
    assert abs(radii[0] - radii[1]) / radii[1] < 5e-3
    assert 1.2 < radii[1] < 1.32


def test_qs_linear_and_zero_mean(oracle):
    rng = np.random.default_rng(4)
    x = rng.random((5, 3)) * 16
    F = rng.standard_normal((5, 3))
    u1 = oracle.qs_velocity((16, 16, 16), 0.0, 1.0, x, F, 1.0)
    u2 = oracle.qs_velocity((16, 16, 16), 0.0, 1.0, x, 2.5 * F, 1.0)
    assert np.abs(u2 - 2.5 * u1).max() <= 1e-13 * np.abs(u1).max()
    assert np.abs(u1.mean(axis=(1, 2, 3))).max() <= 1e-14 * np.abs(u1).max()


def test_qs_fluctuation_dissipation(oracle):
    n, dt, kT, K = 16, 0.01, 1.0, 1500
    pos = (7.3, 8.1, 6.6)
    x = np.array([pos])
    F = np.zeros((1, 3))
    vs = np.array([oracle.interp(oracle.qs_velocity((n, n, n), 0.0, 1.0, x, F, 1.0, 1.0, kT, dt, True, 17, k),
                                 0.0, 1.0, x)[0] for k in range(1, K + 1)])
    for d in range(3):
        m = _mobility(oracle, n, pos, axis=d)
        est = vs[:, d].var() * dt / (2 * kT)
        assert abs(est - m) < 4 * np.sqrt(2.0 / K) * m, (d, est, m)


def test_qs_sim_step_moves_with_interpolated_velocity(oracle):
    from monomers2026_b200 import workloads as W
    wl = W.config(3, kT=0.0, nchains=3, length=10, grid=16, body=0.01)
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    s = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass,
                   ff=ff, integrator=1)
    s.initial()
    x0, F0 = s.x.copy(), s.f.copy()
    s.step(1)
    dx = (p.box_hi - p.box_lo) / p.numMeshPtsPerDir[0]
    u = oracle.qs_velocity(p.numMeshPtsPerDir, p.box_lo, dx, x0, F0, p.mu)
    v = oracle.interp(u, p.box_lo, dx, x0)
    L = p.box_hi - p.box_lo
    d = s.x - (x0 + p.dt * v)
    d -= L * np.round(d / L)
    assert np.abs(d).max() < 1e-13 * L
    assert np.allclose(s.v, v, rtol=0, atol=1e-15 * np.abs(v).max())
    assert np.allclose(s.f, ff.forces(s.x)[0], rtol=0, atol=1e-12)
