"""The reference's own GPU step (oracle/_ref/libselm_refgpu.so: its
cuda/SELM_Eulerian_Period.cu and cuda/SELM_Kernel.cu compiled unchanged for
sm_100a with a stub driver) as a second oracle, at kT = 0 where the step is
deterministic up to the order of its FP64 atomic additions: 16 free monomers
with random initial velocities, no conservative force.  Per step, the
reference GPU path, the FP64 CPU oracle and this library's plain64 form agree
to 1e-12 relative (each field against its maximum).  Also: the cuFFT timing
helper of the bench runs."""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Selm
from oracle import refgpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="oracle/_ref/libselm_refgpu.so not built")]


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


@pytest.mark.parametrize("grid", [16, 30])
def test_reference_gpu_step_matches_oracle_and_plain64(oracle, grid):
    wl = W.config(1, kT=0.0, grid=grid, nchains=16, length=1)
    wl.params.flagStochasticDriving = 0
    wl.v = np.random.default_rng(5).normal(0.0, 0.5, wl.x.shape)
    p = wl.params
    r = refgpu.ReferenceGpuRun(wl)
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass, v=wl.v)
    o.initial()
    g = Selm(p, wl.x, wl.mass, v=wl.v)
    g.initial()
    for k in range(12):
        r.step(1)
        o.step(1)
        g.run(1)
        xr, vr, ur = r.state()
        xg, vg, _ = g.particles()
        ug = g.get_field(0)
        e_ref = max(rel(xr, o.x), rel(vr, o.v), rel(ur, o.u.reshape(ur.shape)))
        e_gpu = max(rel(xg, xr), rel(vg, vr), rel(ug, ur))
        assert e_ref < 1e-12, f"step {k + 1}: reference GPU vs oracle {e_ref:.3e}"
        assert e_gpu < 1e-12, f"step {k + 1}: plain64 vs reference GPU {e_gpu:.3e}"
    assert g.status() == 0
    g.final()
    r.close()


def test_cufft_timing_helper_runs():
    t = refgpu.cufft_time(32, 32, reps=3)
    assert t["r2c_ms"] > 0 and t["c2r_ms"] > 0
