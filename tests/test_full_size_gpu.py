"""The bench workload at its full size (128^3 grid, 1000 FENE+WCA chains of
100 monomers, kT = 1), where the oracle would take minutes a step: properties
that do not depend on the size.

(1) The FP64 spectral form (fused64) and the FP64 reference-structured form
(plain64) are two independent implementations of the same step (spectral
operators against real-space stencils and FFT passes) on the same Philox
stream; each matches the oracle to 1e-11 per step on small grids.  After 5
steps they agree to 1e-10 relative (each field against its maximum).
(2) The FP32 form stays within 1e-5 of FP64 in the velocities (monomer and
fluid) and the forces (1e-9 for positions, which are FP64 in both).
(3) Two runs of the FP32 form are bitwise equal (fixed-point spreading, no
floating-point atomics), and every run ends with a clear status word."""
from dataclasses import replace

import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Selm

pytestmark = pytest.mark.gpu

STEPS = 5


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


@pytest.fixture(scope="module")
def workload():
    return W.config(3)


def _run(wl, form):
    g = Selm(replace(wl.params, form=form), wl.x, wl.mass, v=wl.v, topology=wl.topology)
    g.initial()
    g.run(STEPS)
    x, v, f = g.particles()
    u = g.get_field(0)
    st = g.status()
    g.final()
    return x, v, f, u, st


def test_full_size_forms_agree_and_fp32_is_deterministic(workload):
    assert len(workload.mass) == 100000 and workload.params.numMeshPtsPerDir[0] == 128
    p64 = _run(workload, "plain64")
    f64 = _run(workload, "fused64")
    f32a = _run(workload, "fused32")
    f32b = _run(workload, "fused32")
    for r in (p64, f64, f32a, f32b):
        assert r[4] == 0
    for a, b in zip(f64[:4], p64[:4]):
        assert rel(a, b) < 1e-10
    assert rel(f32a[0], f64[0]) < 1e-9
    for name, a, b in zip(("v", "f", "u"), f32a[1:4], f64[1:4]):
        assert rel(a, b) < 1e-5, f"FP32 {name}: rel err {rel(a, b):.3e}"
    for a, b in zip(f32a[:4], f32b[:4]):
        assert np.array_equal(a, b)
