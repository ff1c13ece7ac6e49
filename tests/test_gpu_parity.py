"""Parity of the CUDA path against the FP64 oracle (run on a B200).

Tolerances (stated per test): FP64 operators 1e-13 relative to the field
maximum; whole FP64 steps 1e-12 relative per step (kT = 0, and kT > 0 with the
same Philox stream in both); FP32 operators 1e-5.
"""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Params, Selm, Topology, op_interp, op_irfft3, op_rfft3, op_spread

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


FFT_DIMS = [(8, 8, 8), (24, 24, 24), (30, 30, 30), (32, 32, 32), (48, 48, 48), (12, 16, 20), (128, 128, 128),
            # odd lengths, and prime factors 11..61 (p-point DFT stages)
            (27, 25, 21), (22, 26, 34), (62, 58, 46), (61, 12, 10)]


@pytest.mark.parametrize("dims", FFT_DIMS)
@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 2e-6)])
def test_fft3_vs_oracle(oracle, dims, prec, tol):
    nx, ny, nz = dims
    rng = np.random.default_rng(nx * 7 + ny)
    a = rng.standard_normal((nz, ny, nx))
    h_ref = oracle.rfft3(a)
    h = op_rfft3(a, prec)
    assert rel(h, h_ref) < tol
    X = rng.standard_normal(h_ref.shape) + 1j * rng.standard_normal(h_ref.shape)  # non-Hermitian planes
    r_ref = oracle.irfft3(X, nx)
    r = op_irfft3(X, nx, prec)
    assert rel(r, r_ref) < tol


def _case(rng, n, M, lo=-3.0):
    L = 0.75 * n
    dx = L / n
    x = lo + rng.random((M, 3)) * L
    x[0] = lo  # on the low face
    x[1] = lo + L  # on the high face (wraps)
    x[2] = lo + dx * np.array([3.0, 3.5, 4.0])  # on nodes: the reference's distance-2 edge case
    return lo, dx, x


@pytest.mark.parametrize("n,M", [(8, 9), (16, 200), (30, 300), (64, 2000)])
@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-5)])
def test_interp_vs_oracle(oracle, n, M, prec, tol):
    rng = np.random.default_rng(n + M)
    lo, dx, x = _case(rng, n, M)
    u = rng.standard_normal((3, n, n, n))
    assert rel(op_interp(u, lo, dx, x, prec), oracle.interp(u, lo, dx, x)) < tol


@pytest.mark.parametrize("n,M", [(8, 9), (16, 200), (30, 300), (64, 2000), (24, 5000)])
@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 1e-5)])
def test_spread_vs_oracle(oracle, n, M, prec, tol):
    rng = np.random.default_rng(n * M)
    lo, dx, x = _case(rng, n, M)
    tf = rng.standard_normal((M, 3))
    base = rng.standard_normal((3, n, n, n))
    assert rel(op_spread(base, lo, dx, x, tf, prec), oracle.spread(base, lo, dx, x, tf)) < tol


def test_spread_dense_cluster_exceeds_one_staging_round(oracle):
    # > 256 monomers inside one tile exercises the chunked candidate staging
    rng = np.random.default_rng(12)
    n = 16
    x = 4.0 + rng.random((900, 3)) * 6.0
    tf = rng.standard_normal((900, 3))
    base = np.zeros((3, n, n, n))
    assert rel(op_spread(base, 0.0, 1.0, x, tf, 64), oracle.spread(base, 0.0, 1.0, x, tf)) < 1e-13


def _oracle_sim(oracle, wl, stochastic=None, noise_mode=0):
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    st = p.flagStochasticDriving if stochastic is None else stochastic
    s = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass, v=wl.v,
                   stochastic=st, seed=p.SELM_Seed, noise_mode=noise_mode, ff=ff)
    s.initial()
    return s


def _gpu_sim(wl):
    s = Selm(wl.params, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    s.initial()
    return s


def _compare_run(oracle, wl, nsteps, tol, every=1):
    o = _oracle_sim(oracle, wl)
    g = _gpu_sim(wl)
    worst = 0.0
    for k in range(nsteps // every):
        o.step(every)
        g.run(every)
        x, v, f = g.particles()
        u = g.get_field(0)
        e = max(rel(x, o.x), rel(v, o.v), rel(u, o.u), rel(f, o.f))
        worst = max(worst, e)
        assert e < tol, f"step {o.nstep}: rel err {e:.3e}"
    assert g.status() == 0
    return worst


def _moving(wl, seed=3, scale=0.3):
    # the random walk starts at the bond rest length; initial velocities make every field non-trivial
    wl.v = np.random.default_rng(seed).normal(0.0, scale, wl.x.shape)
    return wl


def test_plain64_harmonic_chain_kT0(oracle):
    wl = _moving(W.config(1, kT=0.0, grid=16))
    wl.params.flagStochasticDriving = 0
    _compare_run(oracle, wl, 40, 1e-12)


def test_plain64_harmonic_chain_kT1_same_philox(oracle):
    wl = _moving(W.config(1, kT=1.0, grid=16))
    wl.params.flagStochasticDriving = 1
    _compare_run(oracle, wl, 20, 1e-11)


def test_plain64_fene_wca_chains_kT0_body_force(oracle):
    wl = W.config(3, kT=0.0, nchains=4, length=25, grid=24, body=0.01)
    wl.params.flagStochasticDriving = 0
    _compare_run(oracle, wl, 30, 1e-12)


def test_plain64_nucleotide_like_angles_and_ljcut(oracle):
    # 4-bead molecules with harmonic bonds and angles, lj/cut pairs, special 0 0 0,
    # real-unit parameters of the reference's example case
    rng = np.random.default_rng(4)
    nmol = 12
    base = np.array([[0.0, 0.633, 0.0], [0.0, 0.0, 0.0], [0.322, -0.291, 0.0], [-0.322, -0.288, 0.285]])
    x = np.concatenate([base + rng.uniform(-2.5, 2.5, 3) for _ in range(nmol)])
    x = -3.0 + np.mod(x + 3.0, 6.0)
    types = np.tile([1, 2, 3, 4], nmol).astype(np.int32)
    bonds, angles = [], []
    for m in range(nmol):
        o = 4 * m
        bonds += [(1, o, o + 1), (2, o + 1, o + 2), (3, o + 1, o + 3)]
        angles += [(1, o, o + 1, o + 3), (2, o, o + 1, o + 2), (3, o + 2, o + 1, o + 3)]
    eps = [0.542, 0.422, 0.563, 0.637, 0.302, 0.443, 0.517, 0.584, 0.658, 0.732]
    pc = np.zeros((25, 3))
    q = 0
    for i in range(1, 5):
        for j in range(i, 5):
            pc[i * 5 + j] = pc[j * 5 + i] = (1.0, eps[q], 1.0)
            q += 1
    topo = Topology(types=types, ntypes=4, bonds=np.array(bonds, np.int32), bond_style="harmonic",
                    bond_coeff=np.array([[0, 0, 0, 0], [9934.817, 0.7, 0, 0], [2250.785, 0.456, 0, 0],
                                         [4860.383, 0.502, 0, 0]]),
                    angles=np.array(angles, np.int32), angle_style="harmonic",
                    angle_coeff=np.array([[0, 0], [51.084, 99.085], [27.469, 128.857], [37.735, 106.014]]),
                    pair_style="lj/cut", pair_coeff=pc, special_lj=(0.0, 0.0, 0.0))
    mass = np.tile([214.0, 83.0, 217.0, 319.0], nmol)
    p = Params(numMeshPtsPerDir=(30, 30, 30), box_lo=-3.0, box_hi=3.0, rho=493.936086, mu=752.767749,
               KB=0.0083144721451, T=0.0, dt=0.001, flagStochasticDriving=0, SELM_Seed=123456)
    wl = W.Workload("nucleotide", p, x, mass, topo, 30)
    _compare_run(oracle, wl, 30, 1e-12)


def test_plain64_is_deterministic():
    wl = W.config(3, kT=1.0, nchains=6, length=30, grid=32)
    runs = []
    for _ in range(2):
        g = _gpu_sim(wl)
        g.run(10)
        runs.append((g.particles(), g.get_field(0)))
    (x0, v0, f0), u0 = runs[0]
    (x1, v1, f1), u1 = runs[1]
    assert np.array_equal(x0, x1) and np.array_equal(v0, v1) and np.array_equal(u0, u1)


def test_error_word_flags_large_displacement():
    wl = W.config(1, kT=0.0, grid=16)
    wl.params.flagStochasticDriving = 0
    v = np.zeros_like(wl.x)
    v[0, 0] = 2000.0  # |v dt| = 20 > L/2 = 8: the reference only prints (cuda/SELM_Kernel.cu:363)
    g = Selm(wl.params, wl.x, wl.mass, v=v, topology=wl.topology)
    g.initial()
    g.run(1)
    assert g.status() & 0x2


# ---------------------------------------------------------------- fused spectral forms
# FP64 fused: same tolerance as the plain form; FP32 fused: 1e-5 relative (velocity
# error target of the FP32 form), positions in FP64.
@pytest.mark.parametrize("form,tol", [("fused64", 1e-12), ("fused32", 1e-5)])
@pytest.mark.parametrize("kT", [0.0, 1.0])
def test_fused_harmonic_chain_vs_oracle(oracle, form, tol, kT):
    wl = _moving(W.config(1, kT=kT, grid=16, form=form))
    wl.params.flagStochasticDriving = int(kT > 0)
    _compare_run(oracle, wl, 20, tol * (10 if kT > 0 else 1))


@pytest.mark.parametrize("form,tol", [("fused64", 1e-12), ("fused32", 1e-5)])
def test_fused_fene_wca_vs_oracle(oracle, form, tol):
    wl = W.config(3, kT=0.0, nchains=4, length=25, grid=24, body=0.01, form=form)
    wl.params.flagStochasticDriving = 0
    _compare_run(oracle, wl, 20, tol)


@pytest.mark.parametrize("form,tol", [("fused64", 1e-11), ("fused32", 1e-5)])
def test_fused_128_cubed_with_noise(oracle, form, tol):
    """The 128^3 kernels (their own column blocks and block shapes) with the
    thermal noise on: FENE chains against the FP64 oracle, step by step."""
    wl = W.config(3, kT=1.0, nchains=8, length=25, grid=128, form=form)
    _compare_run(oracle, wl, 3, tol)


@pytest.mark.parametrize("grid", [30, 48])
def test_fused64_nonpow2_grid_with_noise(oracle, grid):
    wl = W.config(3, kT=1.0, nchains=3, length=20, grid=grid, form="fused64")
    _compare_run(oracle, wl, 8, 1e-11)


@pytest.mark.parametrize("grid", [22, 26, 27])
@pytest.mark.parametrize("form,tol", [("plain64", 1e-11), ("fused64", 1e-11), ("fused32", 1e-4)])
def test_grids_with_larger_primes_and_odd_grids_with_noise(oracle, grid, form, tol):
    """Grids of 22 = 2 x 11 and 26 = 2 x 13 points per side (p-point DFT
    stages in every FFT) and an odd grid (27, no Nyquist plane), thermal
    noise on: whole steps against the oracle on the same Philox stream."""
    wl = W.config(3, kT=1.0, nchains=3, length=20, grid=grid, form=form)
    _compare_run(oracle, wl, 6, tol)


def test_fused64_exact_noise_mode(oracle):
    wl = _moving(W.config(1, kT=1.0, grid=16, form="fused64"))
    wl.params.noise_mode = "exact"
    o = _oracle_sim(oracle, wl, noise_mode=1)
    g = _gpu_sim(wl)
    o.step(10)
    g.run(10)
    x, v, _ = g.particles()
    assert rel(x, o.x) < 1e-11 and rel(v, o.v) < 1e-11 and rel(g.get_field(0), o.u) < 1e-11


def test_fused_matches_plain64():
    wl = W.config(3, kT=1.0, nchains=5, length=20, grid=32)
    res = {}
    for form in ("plain64", "fused64"):
        wl.params.form = form
        g = _gpu_sim(wl)
        g.run(15)
        res[form] = (g.particles()[1], g.get_field(0))
    assert rel(res["fused64"][0], res["plain64"][0]) < 1e-11
    assert rel(res["fused64"][1], res["plain64"][1]) < 1e-11


def test_fused32_is_deterministic():
    wl = W.config(3, kT=1.0, nchains=6, length=30, grid=32, form="fused32")
    out = []
    for _ in range(2):
        g = _gpu_sim(wl)
        g.run(10)
        out.append((g.particles()[0], g.get_field(0)))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("form", ["fused32", "fused64"])
def test_graph_replay_equals_direct_launches(form):
    # selm_step replays a captured CUDA graph; with per-kernel timing on, the same
    # kernels are launched one by one: both must give identical bits
    wl = W.config(3, kT=1.0, nchains=6, length=30, grid=32, form=form)
    out = []
    for direct in (False, True):
        g = _gpu_sim(wl)
        if direct:
            g.profile(True)
        g.run(12)
        out.append((g.particles(), g.get_field(0)))
    (xa, va, fa), ua = out[0]
    (xb, vb, fb), ub = out[1]
    assert np.array_equal(xa, xb) and np.array_equal(va, vb) and np.array_equal(fa, fb) and np.array_equal(ua, ub)


def test_set_particles_keeps_masses_when_left_out():
    """The per-step host round trip sends positions and velocities only: a
    call with mass = NULL keeps the masses (the run equals one that never
    made the call, bit for bit); a first call without masses is refused."""
    import ctypes as C

    from monomers2026_b200 import _lib
    L = _lib.load()
    dp = C.POINTER(C.c_double)
    wl = W.config(1, kT=1.0, grid=16, form="fused32")
    wl.mass = np.linspace(0.5, 2.0, len(wl.mass))
    a = _gpu_sim(wl)
    b = _gpu_sim(wl)
    a.run(3)
    b.run(3)
    x, v, _ = a.particles()
    x, v = np.ascontiguousarray(x), np.ascontiguousarray(v)
    _lib.check(L.selm_set_particles(a._h, a.M, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None))
    a.run(4)
    b.run(4)
    for p, q in zip(a.particles(), b.particles()):
        assert np.array_equal(p, q)
    h = C.c_void_p()
    _lib.check(L.selm_create(C.byref(wl.params.to_c()), C.byref(h)))
    try:
        assert L.selm_set_particles(h, a.M, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None) != 0
    finally:
        L.selm_destroy(h)


@pytest.mark.parametrize("form,tol", [("plain64", 1e-11), ("fused64", 1e-11), ("fused32", 1e-4)])
@pytest.mark.parametrize("M", [0, 1])
def test_fluid_alone_and_one_monomer_with_noise(oracle, form, tol, M):
    """Edge cases of the monomer side: no monomers at all (the fluid alone,
    thermal forcing on) and a single monomer (no pair partners), against the
    oracle on the same Philox stream."""
    wl = W.config(1, kT=1.0, grid=16, form=form)
    p = wl.params
    x, m = wl.x[:M].copy(), wl.mass[:M].copy()
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, x, m, stochastic=1,
                   seed=p.SELM_Seed)
    o.initial()
    g = Selm(p, x, m)
    g.initial()
    for _ in range(4):
        o.step(2)
        g.run(2)
        assert rel(g.get_field(0), o.u) < tol
        if M:
            xg, vg, _ = g.particles()
            assert rel(xg, o.x) < tol and rel(vg, o.v) < tol
    assert g.status() == 0


def test_monomer_on_the_upper_box_face(oracle):
    """A monomer exactly at box_hi is the periodic image of box_lo: the
    interpolation, spreading and the step give the oracle's results."""
    wl = _moving(W.config(1, kT=0.0, grid=16, form="fused64"))
    wl.params.flagStochasticDriving = 0
    wl.x[0] = [wl.params.box_hi, wl.params.box_lo + 3.0, wl.params.box_hi]
    _compare_run(oracle, wl, 6, 1e-12)


def test_neighbour_list_overflow_is_flagged():
    """More pair partners within reach than a monomer's list holds: the list
    keeps what fits and the status word reports it (0x20), as the force
    kernels then miss pairs."""
    n = 16
    # a 4x4x4 block at spacing 0.45 sigma: the inner monomers have about 50
    # partners within cutoff + skin (1.62 sigma), the list holds 40; the
    # closest pairs stay 0.45 apart, so the forces remain finite
    g1 = np.arange(4) * 0.45
    x = 8.0 + np.stack(np.meshgrid(g1, g1, g1, indexing="ij"), -1).reshape(-1, 3)
    M = len(x)
    pc = np.zeros((4, 3))
    pc[3] = (1.0, 1.0, 2 ** (1 / 6))  # type 1 with itself: WCA
    topo = Topology(types=np.ones(M, np.int32), ntypes=1, pair_style="lj/cut", pair_coeff=pc,
                    special_lj=(0.0, 0.0, 0.0))
    p = Params(numMeshPtsPerDir=(n, n, n), box_lo=0.0, box_hi=float(n), rho=1.0, mu=1.0, KB=1.0, T=0.0, dt=1e-6,
               flagStochasticDriving=0, SELM_Seed=1, form="fused64")
    g = Selm(p, x, np.ones(M), topology=topo)
    g.initial()
    g.run(1)
    assert g.status() & 0x20


def test_set_particles_checks_and_remaps():
    """Non-finite or far positions and non-positive masses are refused and
    leave the simulation's monomers as they were (the positions are checked in
    device staging buffers before they are committed); positions outside the
    box are moved by whole box lengths into [lo, hi), as LAMMPS does at
    setup."""
    import ctypes as C

    from monomers2026_b200 import _lib
    L = _lib.load()
    dp = C.POINTER(C.c_double)
    wl = W.config(1, kT=0.0, grid=16, form="fused32")
    g = _gpu_sim(wl)
    M = g.M
    x0, v0, _ = g.particles()
    for bad in (np.nan, np.inf, -np.inf, 1e12):
        x = np.ascontiguousarray(x0.copy())
        x[M // 2, 1] = bad
        x[0] += 0.125
        v = np.full((M, 3), 0.5)
        assert L.selm_set_particles(g._h, M, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None) == 1  # INVALID
        xg, vg, _ = g.particles()
        assert np.array_equal(xg, x0) and np.array_equal(vg, v0)
    m = np.ones(M)
    m[3] = 0.0
    x = np.ascontiguousarray(x0.copy())
    assert L.selm_set_particles(g._h, M, x.ctypes.data_as(dp), None, m.ctypes.data_as(dp)) == 1
    box = wl.params.box_hi - wl.params.box_lo
    x[0] = [wl.params.box_hi + 0.25, wl.params.box_lo - 0.5, wl.params.box_lo + 3 * box + 0.125]
    _lib.check(L.selm_set_particles(g._h, M, x.ctypes.data_as(dp), None, None))
    got = g.particles()[0]
    assert np.allclose(got[0], [wl.params.box_lo + 0.25, wl.params.box_hi - 0.5, wl.params.box_lo + 0.125])
    assert np.array_equal(got[1:], x0[1:])
    # in-box uploads commit exactly; no velocities means zero velocities
    x1 = np.ascontiguousarray(got.copy())
    x1[5] = wl.params.box_lo + 1.0
    v1 = np.random.default_rng(3).standard_normal((M, 3))
    _lib.check(L.selm_set_particles(g._h, M, x1.ctypes.data_as(dp), v1.ctypes.data_as(dp), None))
    xg, vg, _ = g.particles()
    assert np.array_equal(xg, x1) and np.array_equal(vg, v1)
    _lib.check(L.selm_set_particles(g._h, M, x1.ctypes.data_as(dp), None, None))
    assert np.array_equal(g.particles()[0], x1) and np.all(g.particles()[1] == 0)


@pytest.mark.parametrize("form", ["fused32", "fused64"])
def test_host_round_trip_every_step_is_exact(form):
    """A host round trip every step (positions and velocities uploaded, one
    step, positions, velocities and forces read back), as a host force
    provider runs it, gives bitwise the states of the same simulation stepped
    without it.  After a graph step the read-back waits only for the step's
    monomer state, not for the spread and fluid kernels after it, so this
    also shows that it never reads a state that is not final."""
    import ctypes as C

    from monomers2026_b200 import _lib
    L = _lib.load()
    dp = C.POINTER(C.c_double)
    wl = W.config(2, form=form)
    a, b = _gpu_sim(wl), _gpu_sim(wl)
    M = a.M
    x, v, f = (np.zeros((M, 3)) for _ in range(3))
    _lib.check(L.selm_get_particles(a._h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), f.ctypes.data_as(dp)))
    for _ in range(25):
        _lib.check(L.selm_set_particles(a._h, M, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None))
        _lib.check(L.selm_step(a._h, 1))
        _lib.check(L.selm_get_particles(a._h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), f.ctypes.data_as(dp)))
    b.run(25)
    b.synchronize()
    xb, vb, fb = b.particles()
    assert np.array_equal(x, xb) and np.array_equal(v, vb) and np.array_equal(f, fb)
    assert a.status() == 0 and b.status() == 0
    # a read-back after several steps in one call, then after a full synchronisation
    a.run(3)
    x1, v1, f1 = a.particles()
    a.synchronize()
    x2, v2, f2 = a.particles()
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2) and np.array_equal(f1, f2)


def test_registered_host_arrays_round_trip():
    """Host arrays page-locked through selm_host_register give the same round
    trip, bit for bit, as plain pageable ones; registering twice is not an
    error; unregistering ends it."""
    import ctypes as C

    from monomers2026_b200 import _lib
    from monomers2026_b200.selm import host_register, host_unregister
    L = _lib.load()
    dp = C.POINTER(C.c_double)
    wl = W.config(2, nchains=4, length=50, grid=32, form="fused32")
    sims = [_gpu_sim(wl), _gpu_sim(wl)]
    M = sims[0].M
    bufs = [[np.zeros((M, 3)) for _ in range(3)] for _ in sims]
    for a in bufs[1]:
        host_register(a)
        host_register(a)
    for s, (x, v, f) in zip(sims, bufs):
        _lib.check(L.selm_get_particles(s._h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), f.ctypes.data_as(dp)))
        for _ in range(6):
            _lib.check(L.selm_set_particles(s._h, M, x.ctypes.data_as(dp), v.ctypes.data_as(dp), None))
            _lib.check(L.selm_step(s._h, 1))
            _lib.check(L.selm_get_particles(s._h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), f.ctypes.data_as(dp)))
    for a, b in zip(bufs[0], bufs[1]):
        assert np.array_equal(a, b)
    for a in bufs[1]:
        host_unregister(a)
    with pytest.raises(RuntimeError):
        host_unregister(bufs[1][0])


def test_host_register_refuses_a_partly_registered_range():
    """An array that grew past an earlier registration (same start, larger
    size) is refused, not reported as page-locked; the earlier range itself
    registers again without error."""
    from monomers2026_b200.selm import host_register, host_unregister
    a = np.zeros(1 << 20)
    head = a[: 1 << 18]
    host_register(head)
    with pytest.raises(RuntimeError):
        host_register(a)
    host_register(head)
    host_unregister(head)
    host_register(a)
    host_unregister(a)


def test_host_force_callback_may_add_into_f(oracle):
    """The force array handed to a host provider starts at zero, so a
    provider that adds its forces into f (as LAMMPS' styles do after clearing
    it) steps exactly as one that overwrites f."""
    from monomers2026_b200 import _lib
    wl = W.config(3, kT=0.0, nchains=4, length=25, grid=24, body=0.01, form="fused32")
    wl.params.flagStochasticDriving = 0
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)

    def forces(x):
        f = ff.forces(x)
        return f[0] if isinstance(f, tuple) else f

    def adder(user, natoms, x, v, f):
        xa = np.ctypeslib.as_array(x, (natoms, 3)).copy()
        fa = np.ctypeslib.as_array(f, (natoms, 3))
        fa += forces(xa)
        return 0

    sims = []
    for mode in ("set", "add"):
        s = Selm(p, wl.x, wl.mass, v=wl.v, topology=wl.topology)
        if mode == "set":
            s.set_force_callback(lambda x, v: forces(x))
        else:
            s._cb_keep = _lib.FORCE_FN(adder)
            _lib.check(s._L.selm_set_force_callback(s._h, s._cb_keep, None))
        s.initial()
        sims.append(s)
    for _ in range(4):
        for s in sims:
            s.run(2)
        (x0, v0, f0), (x1, v1, f1) = sims[0].particles(), sims[1].particles()
        assert np.array_equal(x0, x1) and np.array_equal(v0, v1) and np.array_equal(f0, f1)


@pytest.mark.parametrize("form", ["plain64", "fused32"])
def test_host_force_callback_matches_device_force_field(oracle, form):
    """A host force provider (the reference's per-step LAMMPS round trip,
    through the library's page-locked buffers) computing the same FENE + WCA
    forces with the oracle's force field gives the steps of the device force
    field: 1e-12 relative (the two sum the pair forces in another order)."""
    wl = W.config(3, kT=0.0, nchains=4, length=25, grid=24, body=0.01, form=form)
    wl.params.flagStochasticDriving = 0
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    calls = []

    def host_forces(x, v):
        calls.append(1)
        f = ff.forces(x)
        return f[0] if isinstance(f, tuple) else f

    dev = _gpu_sim(wl)
    host = Selm(p, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    host.set_force_callback(host_forces)
    host.initial()
    for _ in range(5):
        dev.run(2)
        host.run(2)
        (xd, vd, fd), (xh, vh, fh) = dev.particles(), host.particles()
        assert rel(xh, xd) < 1e-12 and rel(vh, vd) < 1e-12 and rel(fh, fd) < 1e-12
    assert len(calls) >= 10 and host.status() == 0
