"""The device force field (FENE bonds with their WCA core, WCA pairs from the
Verlet list, the body force) at the full size of the large configuration:
1000 FENE chains of 100 monomers (1e5) in L = 128, against the oracle's force
field (which the reference's own code reproduces bit for bit), at the
initial positions: every monomer's force within 1e-12 of the largest.  The
neighbour list, its cell grid (58 cells per side here) and its scans change
with the system size, so the small-system parity tests do not cover them."""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Selm

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form", ["plain64", "fused32"])
def test_device_forces_match_oracle_at_full_size(oracle, form):
    wl = W.config(3, kT=0.0, body=0.01, form=form)
    wl.params.flagStochasticDriving = 0
    assert len(wl.mass) == 100000
    p = wl.params
    ff = oracle.ForceField(wl.topology.as_dict(), p.box_lo, p.box_hi)
    fo = ff.forces(wl.x)
    fo = fo[0] if isinstance(fo, tuple) else fo
    s = Selm(p, wl.x, wl.mass, topology=wl.topology)
    s.initial()
    _, _, f = s.particles()
    err = np.abs(f - fo).max(1) / np.abs(fo).max()
    bad = np.nonzero(err > 1e-12)[0]
    assert len(bad) == 0, f"{len(bad)} monomers off, e.g. {bad[:5].tolist()}: max {err.max():.3e}"
    assert s.status() == 0
    s.final()
