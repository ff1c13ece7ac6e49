"""CPU checks of the FP64 oracle (the checker of the CUDA path).

The reference ships no golden vectors for this path, so the oracle is pinned
here by the mathematics it restates: FFT against numpy's pocketfft (including
the Hermitian-average behaviour of c2r on non-Hermitian planes), the Peskin
kernel's moment conditions, spread/interpolate adjointness, a divergence-free
projection, the fluid step against an independent numpy restatement, and the
monomer update order.  tests/test_ref_pin.py compares it with the reference's
own CPU code when that has been built.
"""
import numpy as np
import pytest

SIZES = [(8, 8, 8), (12, 10, 6), (24, 24, 24), (30, 30, 30), (16, 32, 8), (7, 5, 9)]


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 7, 8, 12, 24, 30, 32, 48, 49, 64, 96, 128])
def test_fft1_matches_numpy(oracle, n):
    rng = np.random.default_rng(n)
    z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    np.testing.assert_allclose(oracle.fft1(z, -1), np.fft.fft(z), rtol=0, atol=1e-13 * max(1, n))
    np.testing.assert_allclose(oracle.fft1(z, +1), np.fft.ifft(z) * n, rtol=0, atol=1e-13 * max(1, n))


@pytest.mark.parametrize("dims", SIZES)
def test_fft3_matches_numpy(oracle, dims):
    nx, ny, nz = dims
    rng = np.random.default_rng(sum(dims))
    a = rng.standard_normal((nz, ny, nx))
    h = oracle.rfft3(a)
    np.testing.assert_allclose(h, np.fft.rfftn(a), rtol=0, atol=1e-12 * a.size ** 0.5)
    X = rng.standard_normal(h.shape) + 1j * rng.standard_normal(h.shape)  # non-Hermitian planes
    r = oracle.irfft3(X, nx)
    ref = np.fft.irfftn(X, s=(nz, ny, nx), axes=(0, 1, 2)) * (nx * ny * nz)
    np.testing.assert_allclose(r, ref, rtol=0, atol=1e-12 * a.size ** 0.5)


def test_peskin_moments(oracle):
    # sum_j phi(r - j) = 1, sum_j (r - j) phi(r - j) = 0, sum_j phi^2 = 3/8
    for r in np.linspace(0.0, 0.999, 37):
        pts = [r + 1, r, r - 1, r - 2]
        w = np.array([oracle.phi(abs(t)) for t in pts])
        assert abs(w.sum() - 1) < 1e-14
        assert abs(np.dot(pts, w)) < 1e-14
        assert abs((w ** 2).sum() - 3 / 8) < 1e-14


def _rand_case(rng, dims, M, L=None):
    nx, ny, nz = dims
    L = float(nx) if L is None else L
    lo = -0.3 * L
    dx = L / nx
    x = lo + rng.random((M, 3)) * L
    return lo, dx, x


@pytest.mark.parametrize("dims", [(8, 8, 8), (16, 16, 16), (12, 12, 12)])
def test_spread_interp_adjoint(oracle, dims):
    rng = np.random.default_rng(3)
    nx, ny, nz = dims
    lo, dx, x = _rand_case(rng, dims, 17)
    u = rng.standard_normal((3, nz, ny, nx))
    tf = rng.standard_normal((17, 3))
    g = oracle.interp(u, lo, dx, x)
    s = oracle.spread(np.zeros((3, nz, ny, nx)), lo, dx, x, tf)  # = -Lambda tf
    assert abs(np.sum(g * tf) + np.sum(s * u)) < 1e-11 * np.abs(g * tf).sum()


def test_interp_of_constant_and_linear_field(oracle):
    rng = np.random.default_rng(5)
    dims = (16, 16, 16)
    lo, dx, x = _rand_case(rng, dims, 11)
    u = np.ones((3, 16, 16, 16)) * np.array([1.5, -2.0, 0.25])[:, None, None, None]
    np.testing.assert_allclose(oracle.interp(u, lo, dx, x), np.tile([1.5, -2.0, 0.25], (11, 1)), atol=1e-13)


def _np_fluid(u, f, dx, mu, rho, dt):
    """Independent numpy restatement (spectral) of mpi/SELM_Eulerian_Period.cpp:86-102."""
    _, nz, ny, nx = u.shape
    lap = sum(np.roll(u, s, axis=a) for a in (1, 2, 3) for s in (1, -1)) - 6 * u
    us = u + (mu * lap / dx ** 2 * dt + f) / rho
    p = sum(np.roll(us[d], -1, axis=2 - d) - us[d] for d in range(3)) / dx
    ph = np.fft.rfftn(p)
    kx = 2 * np.pi * np.arange(nx // 2 + 1) / nx
    ky = 2 * np.pi * np.arange(ny) / ny
    kz = 2 * np.pi * np.arange(nz) / nz
    sym = (2 * (np.cos(kz)[:, None, None] - 1) + 2 * (np.cos(ky)[None, :, None] - 1)
           + 2 * (np.cos(kx)[None, None, :] - 1)) / dx ** 2
    sym[0, 0, 0] = 1.0
    ph = ph / sym
    ph[0, 0, 0] = 0
    p = np.fft.irfftn(ph, s=(nz, ny, nx), axes=(0, 1, 2))
    out = us.copy()
    for d in range(3):
        out[d] -= (p - np.roll(p, 1, axis=2 - d)) / dx
    out -= out.mean(axis=(1, 2, 3), keepdims=True)
    return out


@pytest.mark.parametrize("dims", [(8, 8, 8), (12, 12, 12), (16, 16, 16)])
def test_fluid_step_matches_numpy(oracle, dims):
    rng = np.random.default_rng(11)
    nx, ny, nz = dims
    u = rng.standard_normal((3, nz, ny, nx))
    f = rng.standard_normal((3, nz, ny, nx))
    got = oracle.fluid_run(u, f, 0.7, 0.9, 1.3, 0.05)
    ref = _np_fluid(u, f, 0.7, 0.9, 1.3, 0.05)
    np.testing.assert_allclose(got, ref, atol=1e-12 * np.abs(ref).max())


def test_projection_is_divergence_free(oracle):
    rng = np.random.default_rng(2)
    u = rng.standard_normal((3, 12, 12, 12))
    out = oracle.fluid_run(u, np.zeros_like(u), 1.0, 0.0, 1.0, 0.01)
    div = sum(np.roll(out[d], -1, axis=2 - d) - out[d] for d in range(3))
    assert np.abs(div).max() < 1e-12 * np.abs(out).max()
    assert np.abs(out.mean(axis=(1, 2, 3))).max() < 1e-14


def test_noise_ref_compat_is_hermitian_average(oracle):
    # the c2r of the reference's half-spectrum draw keeps (X + conj X')/2 on the x=0 plane
    dims = (8, 8, 8)
    rng = np.random.default_rng(4)
    xi = (rng.standard_normal((3, 8, 8, 5)) + 1j * rng.standard_normal((3, 8, 8, 5)))
    xi_flat = np.ascontiguousarray(xi).view(np.float64)
    f0 = oracle.noise_from_normals(dims, 1.0, 1.0, xi_flat, 0)
    f1 = oracle.noise_from_normals(dims, 1.0, 1.0, xi_flat, 1)
    h0 = np.fft.rfftn(f0[0]) / 512
    h1 = np.fft.rfftn(f1[0]) / 512
    # interior planes identical, x=0 plane (non-self-conjugate modes) scaled by sqrt(2)
    np.testing.assert_allclose(h0[:, :, 1:4], h1[:, :, 1:4], atol=1e-13)
    m = np.abs(h0[:, :, 0]) > 1e-10
    for k in (0, 4):
        for j in (0, 4):
            m[k, j] = False  # self-conjugate modes keep their variance
    np.testing.assert_allclose(np.abs(h1[:, :, 0][m]) / np.abs(h0[:, :, 0][m]), np.sqrt(2), rtol=1e-10)


def test_philox_streams_are_deterministic(oracle):
    a = oracle.fluid_normals(7, 3, (8, 8, 8))
    b = oracle.fluid_normals(7, 3, (8, 8, 8))
    c = oracle.fluid_normals(7, 4, (8, 8, 8))
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    z = np.concatenate([oracle.fluid_normals(s, 1, (16, 16, 16)).ravel().view(np.float64) for s in range(4)])
    assert abs(z.mean()) < 0.01 and abs(z.var() - 1) < 0.01


def test_lagrangian_update_order(oracle):
    # x advances with the old velocity, v with the new impulse (cuda/SELM_Kernel.cu:355-371)
    from oracle.pyoracle import lib
    rng = np.random.default_rng(9)
    dims = (8, 8, 8)
    u = rng.standard_normal((3, 8, 8, 8))
    x = rng.random((3, 3)) * 8
    v = rng.standard_normal((3, 3))
    f = rng.standard_normal((3, 3))
    m = np.array([1.0, 2.0, 0.5])
    fg = np.zeros((3, 8, 8, 8))
    x0, v0, f0 = x.copy(), v.copy(), f.copy()
    dt, ups = 0.01, 0.3
    g = oracle.interp(u, 0.0, 1.0, x)
    import ctypes as C
    lib().orc_lagrangian_update(x.ravel(), v.ravel(), f.ravel(), m, u.ravel(), fg.ravel(), 8, 8, 8, 0.0, 8.0, 1.0, dt,
                                ups, 0.0, None, 3)
    tf = -ups * (v0 - g) * dt + dt * f0
    np.testing.assert_allclose(f, tf / dt, rtol=1e-14)
    xe = x0 + v0 * dt
    xe = np.where(xe > 8, xe - 8, np.where(xe < 0, xe + 8, xe))
    np.testing.assert_allclose(x, xe, rtol=1e-15)
    np.testing.assert_allclose(v, v0 + tf / m[:, None], rtol=1e-14)
    del C, dims


def test_forces_newton_third_law_and_gradient(oracle):
    from monomers2026_b200 import workloads as W
    rng = np.random.default_rng(1)
    x = W.random_walk_chains(3, 12, 16.0, 0.0, rng, min_sep=0.95)
    topo = W.fene_wca_topology(3, 12).as_dict()
    ff = oracle.ForceField(topo, 0.0, 16.0)
    f, warn = ff.forces(x)
    assert warn == 0
    assert np.abs(f.sum(axis=0)).max() < 1e-10 * np.abs(f).max()
