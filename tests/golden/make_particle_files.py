"""Generates particle_files_kT0.npz (run where oracle/_ref is built).

The reference's particleX/V/F.dat output ("%g %g %g" per monomer after every
saveSkipSimulationData-th step; mpi/SELM_Lagrangian_LAMMPS.cpp:79-82,
280-300), written by the reference's own CPU code (oracle/_ref) on the golden
NucleotideMonomer case (tests/golden/nucleotide_kT0.npz, thermal driving off)
with saveSkipSimulationData 10 and 20 steps: writes after steps 10 and 20.  Stored: the
values parsed from the three files, [write][monomer][3].

Usage: python tests/golden/make_particle_files.py
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

STEPS, SKIP = 20, 10


def write_case_with_files(tmp):
    from test_golden import golden, golden_params, golden_topology

    from monomers2026_b200.casefiles import write_case
    d = golden()
    write_case(tmp, golden_params(d), d["x0"], d["mass_per_type"], golden_topology(d), STEPS)
    with open(os.path.join(tmp, "Model.SELM"), "a") as f:
        f.write(f"saveSkipSimulationData {SKIP}\nwriteParticalX 1\nwriteParticalV 1\nwriteParticalF 1\n")
    return len(d["types"])


def read_files(d, M):
    out = {}
    for k in "XVF":
        a = np.loadtxt(os.path.join(d, f"particle{k}.dat")).reshape(-1, M, 3)
        out[k] = a
    return out


def main():
    from oracle import refdriver
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        M = write_case_with_files(tmp)
        os.chdir(tmp)  # the reference writes the files into the working directory
        try:
            r = refdriver.ReferenceRun(tmp)
            r.step(STEPS)
            r.close()
        finally:
            os.chdir(cwd)
        files = read_files(tmp, M)
    assert all(v.shape == (STEPS // SKIP, M, 3) for v in files.values())
    out = os.path.join(HERE, "particle_files_kT0.npz")
    np.savez_compressed(out, X=files["X"], V=files["V"], F=files["F"], steps=STEPS, skip=SKIP)
    print("wrote", out)


if __name__ == "__main__":
    main()
