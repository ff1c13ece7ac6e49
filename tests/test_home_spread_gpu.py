"""The FP32 spread by home tiles (k_spread_home and its folds), which FP32
simulations of 16384 monomers or more use, on grids that reach each of its
paths: tiles that divide the grid (the column fold), partial last tiles of at
least 4 cells and of fewer (the two general folds), one tile per axis (boxes
that wrap onto themselves), and tiles of more than 2048 monomers (the
two-word split path).  Free monomers with random velocities at kT = 0, three
steps: the FP32 form's positions agree with the FP64 form's to 1e-9 and its
monomer and fluid velocities to 1e-5 (relative to each field's maximum), and
two FP32 runs are bitwise equal."""
from dataclasses import replace

import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Selm

pytestmark = pytest.mark.gpu


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def _run(wl, v0, form, steps=3):
    s = Selm(replace(wl.params, form=form), wl.x, wl.mass, v=v0, topology=wl.topology)
    s.initial()
    s.run(steps)
    x, v, _ = s.particles()
    u = s.get_field(0)
    assert s.status() == 0
    s.final()
    return x, v, u


# (grid, monomers): 64 divides into tiles; 36 leaves last tiles of 4 cells,
# 34 of 2; 24 puts ~2900 monomers in a tile; 16 has one tile along x and z
@pytest.mark.parametrize("n,M", [(64, 20000), (36, 20000), (34, 20000), (24, 20000), (16, 16384)])
def test_home_spread_fp32_matches_fp64_and_repeats(n, M):
    wl = W.config(1, kT=0.0, grid=n, nchains=M, length=1, seed=77 + n)
    wl.params.flagStochasticDriving = 0
    assert len(wl.mass) == M
    v0 = np.random.default_rng(n).normal(0.0, 0.3, wl.x.shape)
    x64, v64, u64 = _run(wl, v0, "fused64")
    x32, v32, u32 = _run(wl, v0, "fused32")
    errs = {"x": rel(x32, x64), "v": rel(v32, v64), "u": rel(u32, u64)}
    assert errs["x"] < 1e-9 and errs["v"] < 1e-5 and errs["u"] < 1e-5, errs
    x32b, v32b, u32b = _run(wl, v0, "fused32")
    assert np.array_equal(x32, x32b) and np.array_equal(v32, v32b) and np.array_equal(u32, u32b)
