"""Pins the FP64 oracle to the reference's own CPU code.

oracle/_ref/libselm_ref.so is the reference's mpi/SELM.cpp,
SELM_Eulerian_Period.cpp and SELM_Lagrangian_LAMMPS.cpp compiled unchanged
(oracle/ref.mk) against single-rank MPI / FFTW-MPI / LAMMPS shims.  At kT = 0
the oracle restatement must reproduce it bit for bit, step by step, on inputs
written as a reference case directory (Model.SELM, LAMMPS script and data);
at kT > 0 (different random streams) their statistics must agree.
"""
import numpy as np
import pytest

from oracle import refdriver

pytestmark = pytest.mark.skipif(not refdriver.available(), reason="oracle/_ref not built (needs the reference source)")


def _run_pair(oracle, wl, nsteps):
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass, v=wl.v,
                   ff=ff)
    o.initial()
    r = refdriver.ReferenceRun(wl, nsteps=nsteps)
    yield o, r
    for _ in range(nsteps):
        o.step()
        r.step()
        yield o, r


@pytest.mark.parametrize("case", ["harmonic", "fene_body", "angles_ljcut"])
def test_oracle_is_bit_exact_with_reference_cpu_code(oracle, case):
    from monomers2026_b200 import workloads as W
    if case == "harmonic":
        wl = W.config(1, kT=0.0, grid=16)
    elif case == "fene_body":
        wl = W.config(3, kT=0.0, nchains=4, length=25, grid=24, body=0.01)
    else:
        wl = _nucleotide_like()
    wl.params.flagStochasticDriving = 0
    wl.v = np.random.default_rng(3).normal(0.0, 0.3, wl.x.shape)
    for o, r in _run_pair(oracle, wl, 15):
        x, v, f, u = r.state()
        assert np.array_equal(x, o.x) and np.array_equal(v, o.v)
        assert np.array_equal(f, o.f) and np.array_equal(u, o.u)


def test_reference_noise_matches_oracle_statistically(oracle):
    """kT > 0: the reference draws RanMars normals and the oracle Philox ones,
    so only statistics compare.  From rest, after six steps, the RMS of each
    fluid-velocity component (32^3 cells) agrees within 3% (measured: 1.008,
    1.014, 0.998), and the monomers' velocity RMS within 25% (20 monomers,
    60 samples; measured 0.90).  An error in the
    thermal forcing's amplitude or in its three-field inverse transform shows
    up here as a factor, not a few percent."""
    from monomers2026_b200 import workloads as W
    wl = W.config(1, kT=1.0, grid=32)
    p = wl.params
    r = refdriver.ReferenceRun(wl, nsteps=6)
    r.step(6)
    _, v_ref, _, u_ref = r.state()
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass,
                   stochastic=1, seed=p.SELM_Seed, ff=ff)
    o.initial()
    o.step(6)
    u_o = o.u.reshape(u_ref.shape)
    assert np.isfinite(u_ref).all()
    for d in range(3):
        a, b = u_ref[d].std(), u_o[d].std()
        assert abs(a / b - 1) < 0.03, (d, a, b)
    assert abs(v_ref.std() / o.v.std() - 1) < 0.25


def _nucleotide_like(nmol=10, seed=4):
    from monomers2026_b200 import workloads as W
    from monomers2026_b200.selm import Params, Topology
    rng = np.random.default_rng(seed)
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
    return W.Workload("nucleotide", p, x, mass, topo, 30)
