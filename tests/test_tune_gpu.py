"""Tuning knobs and the autotuner of the fused forms (B200).

The four-step split only reorders the FFT arithmetic (results agree to the
rounding of the form: 1e-12 relative in FP64, 1e-5 in FP32, and FP64 still
matches the oracle); the z-kernel occupancy cap changes nothing but the
schedule (results equal bit for bit).
"""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.autotune import four_step_splits, tune
from monomers2026_b200.selm import TUNE_FFT_SPLIT, TUNE_Z_BLOCKS, Selm, tune_default

pytestmark = pytest.mark.gpu


def rel(a, b):
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


def _run(wl, nsteps, **knobs):
    s = Selm(wl.params, wl.x, wl.mass, v=wl.v, topology=wl.topology)
    for k, v in knobs.items():
        s.tune({"split": TUNE_FFT_SPLIT, "zb": TUNE_Z_BLOCKS}[k], v)
    s.initial()
    s.run(nsteps)
    x, v, f = s.particles()
    u = s.get_field(0)
    s.final()
    return x, v, u


def test_splits_of_the_sizes():
    assert four_step_splits(128) == (16, 16)
    assert four_step_splits(96) == (16, 12)
    assert four_step_splits(64) == (16, 8)
    assert four_step_splits(48) == (16, 8)
    assert four_step_splits(32) == (16, 8)


@pytest.mark.parametrize("form,tol", [("fused64", 1e-12), ("fused32", 1e-5)])
@pytest.mark.parametrize("grid", [32, 48])
def test_fft_split_changes_only_rounding(oracle, form, tol, grid):
    wl = W.config(3, kT=1.0, nchains=3, length=20, grid=grid, form=form)
    a = _run(wl, 8, split=0)
    b = _run(wl, 8, split=1)
    for p, q in zip(a, b):
        assert rel(p, q) < tol


def test_z_blocks_cap_changes_nothing():
    wl = W.config(3, kT=1.0, nchains=3, length=20, grid=32, form="fused32")
    ref = _run(wl, 6, zb=0)
    for zb in (2, 3, 4):
        got = _run(wl, 6, zb=zb)
        assert all(np.array_equal(p, q) for p, q in zip(ref, got)), zb


def test_defaults_apply_to_later_simulations():
    tune_default(24, 32, TUNE_FFT_SPLIT, 1)
    tune_default(24, 32, TUNE_Z_BLOCKS, 2)
    wl = W.config(3, kT=1.0, nchains=2, length=10, grid=24, form="fused32")
    s = Selm(wl.params, wl.x, wl.mass, topology=wl.topology)
    assert s.tuned(TUNE_FFT_SPLIT) == 1 and s.tuned(TUNE_Z_BLOCKS) == 2
    s.final()
    tune_default(24, 32, TUNE_FFT_SPLIT, 0)
    tune_default(24, 32, TUNE_Z_BLOCKS, 3)


def test_autotuner_records_its_choice():
    wl = W.config(3, kT=1.0, nchains=3, length=20, grid=32, form="fused32")
    out = tune(wl, steps=3, warmup=1)
    assert set(out["choice"]) == {"fft_split", "z_blocks_per_sm"}
    assert len(out["ms"]) == 8
    s = Selm(wl.params, wl.x, wl.mass, topology=wl.topology)
    assert s.tuned(TUNE_FFT_SPLIT) == out["choice"]["fft_split"]
    assert s.tuned(TUNE_Z_BLOCKS) == out["choice"]["z_blocks_per_sm"]
    s.final()
