"""The reference's own GPU step (oracle/_ref/libselm_refgpu.so: its
cuda/SELM_Eulerian_Period.cu and cuda/SELM_Kernel.cu compiled unchanged for
sm_100a with a stub driver) as a second oracle, at kT = 0 where the step is
deterministic up to the order of its FP64 atomic additions: 16 free monomers
with random initial velocities, no conservative force.  Per step, the
reference GPU path, the FP64 CPU oracle and this library's plain64 form agree
to 1e-12 relative (each field against its maximum).

The reference's Eulerian_Period::initial can run once per process only (it
raises the printf FIFO limit, which CUDA refuses after a kernel that prints
has run, and its next checked call then exits the process), so each case
runs in a child process.  Also: the cuFFT timing helper of the bench runs."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import refgpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refgpu.available(), reason="oracle/_ref/libselm_refgpu.so not built")]

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def _case(grid: int) -> dict:
    from monomers2026_b200 import workloads as W
    from monomers2026_b200.selm import Selm
    from oracle import pyoracle as oracle
    wl = W.config(1, kT=0.0, grid=grid, nchains=16, length=1)
    wl.params.flagStochasticDriving = 0
    wl.v = np.random.default_rng(5).normal(0.0, 0.5, wl.x.shape)
    p = wl.params
    r = refgpu.ReferenceGpuRun(wl)
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, wl.x, wl.mass, v=wl.v)
    o.initial()
    g = Selm(p, wl.x, wl.mass, v=wl.v)
    g.initial()
    e_ref = e_gpu = 0.0
    for _ in range(12):
        r.step(1)
        o.step(1)
        g.run(1)
        xr, vr, ur = r.state()
        xg, vg, _ = g.particles()
        ug = g.get_field(0)
        e_ref = max(e_ref, rel(xr, o.x), rel(vr, o.v), rel(ur, o.u.reshape(ur.shape)))
        e_gpu = max(e_gpu, rel(xg, xr), rel(vg, vr), rel(ug, ur))
    out = {"ref_vs_oracle": e_ref, "plain64_vs_ref": e_gpu, "status": g.status()}
    g.final()
    r.close()
    return out


@pytest.mark.parametrize("grid", [16, 30])
def test_reference_gpu_step_matches_oracle_and_plain64(grid):
    env = dict(os.environ, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    res = subprocess.run([sys.executable, os.path.abspath(__file__), str(grid)], capture_output=True, text=True,
                         env=env, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    out = json.loads(res.stdout.strip().splitlines()[-1])
    assert out["status"] == 0
    assert out["ref_vs_oracle"] < 1e-12, out
    assert out["plain64_vs_ref"] < 1e-12, out


def test_cufft_timing_helper_runs():
    t = refgpu.cufft_time(32, 32, reps=3)
    assert t["r2c_ms"] > 0 and t["c2r_ms"] > 0


if __name__ == "__main__":
    print(json.dumps(_case(int(sys.argv[1]))))
