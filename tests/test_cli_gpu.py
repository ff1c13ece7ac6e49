"""The selm_b200 executable as a drop-in for the reference's executable on a
case directory: particleX/V/F.dat ("%g %g %g" per monomer after every
saveSkipSimulationData-th step) against the files the reference's own CPU
code writes on the golden NucleotideMonomer case (thermal driving off;
tests/golden/particle_files_kT0.npz, made by make_particle_files.py).
Tolerance: the printed six significant digits (1e-5 of each file's largest
value; FP32 form 1e-4).  F is the force array as the update leaves it,
(t_f + dt f_before) / dt, not the recomputed conservative force."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from test_golden import golden, golden_params, golden_topology

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(os.path.dirname(HERE), "monomers2026_b200", "lib", "selm_b200")
FIX = os.path.join(HERE, "golden", "particle_files_kT0.npz")


@pytest.mark.parametrize("form,tol", [("plain64", 1e-5), ("fused64", 1e-5), ("fused32", 1e-4)])
def test_cli_particle_files_match_reference(form, tol):
    from monomers2026_b200.casefiles import write_case
    ref = np.load(FIX)
    d = golden()
    M = len(d["types"])
    steps, skip = int(ref["steps"]), int(ref["skip"])
    with tempfile.TemporaryDirectory() as tmp:
        write_case(tmp, golden_params(d, form), d["x0"], d["mass_per_type"], golden_topology(d), steps)
        with open(os.path.join(tmp, "Model.SELM"), "a") as f:
            f.write(f"form {form}\nsaveSkipSimulationData {skip}\nwriteParticalX 1\nwriteParticalV 1\n"
                    "writeParticalF 1\n")
        r = subprocess.run([EXE, tmp], cwd=tmp, capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        for k in "XVF":
            ours = np.loadtxt(os.path.join(tmp, f"particle{k}.dat")).reshape(-1, M, 3)
            want = ref[k]
            assert ours.shape == want.shape, k
            err = np.abs(ours - want).max() / np.abs(want).max()
            assert err < tol, (k, err)
