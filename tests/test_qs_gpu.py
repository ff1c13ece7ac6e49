"""The quasi-steady (overdamped) fused forms against the FP64 oracle (B200).

Same Philox counters in both, so kT > 0 runs compare deterministically.
Tolerances: fused64 1e-12 relative per step at kT = 0, 1e-11 at kT > 0;
fused32 1e-5.  The generic (non-four-step) spectral kernels are covered by
a 20^3 grid.  The plain form has no quasi-steady variant and must refuse it.
"""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Selm

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def _pair(oracle, wl):
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass, v=wl.v,
                   stochastic=p.flagStochasticDriving, seed=p.SELM_Seed, ff=ff, integrator=1)
    o.initial()
    g = Selm(p, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    g.initial()
    return o, g


def _run(oracle, wl, nsteps, tol):
    wl.params.integrator = "quasi_steady"
    o, g = _pair(oracle, wl)
    for _ in range(nsteps):
        o.step(1)
        g.run(1)
        x, v, f = g.particles()
        e = max(rel(x, o.x), rel(v, o.v), rel(f, o.f), rel(g.get_field(0), o.u))
        assert e < tol, f"step {o.nstep}: rel err {e:.3e}"
    assert g.status() == 0


@pytest.mark.parametrize("form,tol", [("fused64", 1e-12), ("fused32", 1e-5)])
def test_qs_fene_wca_body_force_kT0(oracle, form, tol):
    wl = W.config(3, kT=0.0, nchains=4, length=25, grid=24, body=0.01, form=form)
    wl.params.flagStochasticDriving = 0
    _run(oracle, wl, 20, tol)


def test_qs_fused64_harmonic_chain_kT1_same_philox(oracle):
    wl = W.config(1, kT=1.0, grid=16, form="fused64")
    wl.params.flagStochasticDriving = 1
    _run(oracle, wl, 10, 1e-11)


def test_qs_fused64_generic_grid_kT1(oracle):
    wl = W.config(3, kT=1.0, nchains=3, length=15, grid=20, form="fused64")
    wl.params.flagStochasticDriving = 1
    _run(oracle, wl, 6, 1e-11)


def test_qs_fused32_kT1_close_to_fp64(oracle):
    wl = W.config(1, kT=1.0, grid=32, form="fused32")
    wl.params.flagStochasticDriving = 1
    _run(oracle, wl, 10, 1e-4)


def test_qs_plain_form_is_refused():
    wl = W.config(1, kT=0.0, grid=16, form="plain64")
    wl.params.integrator = "quasi_steady"
    with pytest.raises(Exception):
        Selm(wl.params, wl.x, wl.mass, topology=wl.topology)


@pytest.mark.parametrize("M", [0, 1])
def test_qs_fluid_alone_and_one_monomer(oracle, M):
    """The quasi-steady form with no monomers (the thermal forcing alone) and
    with one free monomer, against the oracle on the same Philox stream."""
    wl = W.config(1, kT=1.0, grid=16, form="fused64")
    p = wl.params
    p.integrator = "quasi_steady"
    x, m = wl.x[:M].copy(), wl.mass[:M].copy()
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, x, m, stochastic=1,
                   seed=p.SELM_Seed, integrator=1)
    o.initial()
    g = Selm(p, x, m)
    g.initial()
    for _ in range(3):
        o.step(2)
        g.run(2)
        assert rel(g.get_field(0), o.u) < 1e-11
        if M:
            assert rel(g.particles()[0], o.x) < 1e-11
    assert g.status() == 0
