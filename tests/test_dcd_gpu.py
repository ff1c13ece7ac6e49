"""The selm_b200 executable writes the LAMMPS script's "dump ID group dcd N
file" as a DCD trajectory: frames at step 0 and every N steps, holding the
positions of the reference's NucleotideMonomer example run (tests/golden) as
float32 (tolerance: float32 rounding of the 1e-12-exact FP64 path), up to
whole box lengths (positions are wrapped into the box, as LAMMPS does)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from test_golden import golden, golden_params, golden_topology

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "monomers2026_b200", "lib", "selm_b200")


@pytest.mark.parametrize("form", ["plain64", "fused64"])
def test_cli_dump_dcd(form):
    from monomers2026_b200.casefiles import write_case
    from monomers2026_b200.dcd import read_dcd
    d = golden()
    p = golden_params(d, form)
    with tempfile.TemporaryDirectory() as tmp:
        write_case(tmp, p, d["x0"], d["mass_per_type"], golden_topology(d), 30)
        with open(tmp + "/Model.SELM", "a") as f:
            f.write(f"form {form}\n")
        with open(tmp + "/Model.LAMMPS_script", "a") as f:
            f.write("dump 1 all dcd 10 traj.dcd\n")
        r = subprocess.run([EXE, tmp], cwd=tmp, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        t = read_dcd(tmp + "/traj.dcd")
    M = len(d["types"])
    assert (t["nset"], t["istart"], t["nsavc"], t["nstep"], t["natoms"]) == (4, 0, 10, 30, M)
    assert abs(t["dt"] - np.float32(p.dt)) == 0
    L = p.box_hi - p.box_lo
    assert np.allclose(t["cells"], [L, 0, L, 0, 0, L])
    for k, s in ((0, 0), (1, 10), (3, 30)):
        # the same point of the periodic box (an initial position on the boundary may be wrapped)
        dd = t["xyz"][k].astype(np.float64) - d[f"x{s}"]
        dd -= L * np.round(dd / L)
        assert np.abs(dd).max() <= 1e-6 * max(1.0, np.abs(d[f"x{s}"]).max())
