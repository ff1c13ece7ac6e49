"""Reference case directories: Model.SELM + Model.LAMMPS_script + data file.

The reference runs from a directory holding ``Model.SELM`` (ParmParse keys,
cuda/SELM.cu:17-48) and ``Model.LAMMPS_script`` (read by the embedded LAMMPS,
cuda/SELM_Lagrangian_LAMMPS.cu:21-28), which reads a LAMMPS data file.  This
module writes such a directory from a workload (the C++ reader is
``selm_create_from_files``), so the same inputs drive this library and the
reference's own code.
"""
from __future__ import annotations

import os

import numpy as np

from .selm import Params, Topology

BOND_NAME = {"harmonic": "harmonic", "fene": "fene"}


def _f(v) -> str:
    """Shortest round-trip decimal of a float (exact when read back)."""
    return repr(float(v))


def write_case(dirpath: str, params: Params, x: np.ndarray, mass_per_type: np.ndarray, topo: Topology,
               nsteps: int, v: np.ndarray | None = None, data_name: str = "Model.LAMMPS_read_data") -> str:
    """Write a case directory; masses are per atom type (index 1..ntypes)."""
    os.makedirs(dirpath, exist_ok=True)
    p = params
    with open(os.path.join(dirpath, "Model.SELM"), "w") as f:
        f.write("#Required Parameters\n")
        f.write(f"mu {_f(p.mu)}\nrho {_f(p.rho)}\nKB {_f(p.KB)}\nT {_f(p.T)}\n")
        f.write("EulerianType Eulerian_Period\nLagrangianType Lagrangian_LAMMPS\n")
        f.write(f"nsteps {int(nsteps)}\n")
        f.write("#Optional Parameters\n")
        f.write(f"flagStochasticDriving {int(p.flagStochasticDriving)}\n")
        f.write(f"SELM_Seed {int(p.SELM_Seed)}\n")
        n = p.numMeshPtsPerDir
        f.write(f"numMeshPtsPerDir {n[0]} {n[1]} {n[2]}\n")
    t = topo
    M = len(x)
    with open(os.path.join(dirpath, "Model.LAMMPS_script"), "w") as f:
        f.write("units real\nboundary p p p\natom_style angle\n")
        f.write(f"read_data {data_name}\n")
        if t.bond_style != "none" and len(t.bonds):
            f.write(f"bond_style {BOND_NAME[t.bond_style]}\n")
            for bt in range(1, len(t.bond_coeff)):
                c = t.bond_coeff[bt]
                vals = c[:2] if t.bond_style == "harmonic" else c[:4]
                f.write(f"bond_coeff {bt} " + " ".join(_f(q) for q in vals) + "\n")
        if t.angle_style != "none" and len(t.angles):
            f.write("angle_style harmonic\n")
            for at in range(1, len(t.angle_coeff)):
                c = t.angle_coeff[at]
                f.write(f"angle_coeff {at} {_f(c[0])} {_f(c[1])}\n")
        if t.pair_style == "lj/cut":
            nt = t.ntypes
            pc = np.asarray(t.pair_coeff).reshape(nt + 1, nt + 1, 3)
            f.write(f"pair_style lj/cut {_f(pc[1:, 1:, 2].max())}\n")
            for i in range(1, nt + 1):
                for j in range(i, nt + 1):
                    e, s_, rc = pc[i, j]
                    f.write(f"pair_coeff {i} {j} {_f(e)} {_f(s_)} {_f(rc)}\n")
        sl = t.special_lj
        f.write(f"special_bonds lj {_f(sl[0])} {_f(sl[1])} {_f(sl[2])}\n")
        bf = [float(q) for q in t.body_force]
        if any(bf):
            f.write(f"fix body all addforce {_f(bf[0])} {_f(bf[1])} {_f(bf[2])}\n")
        f.write(f"timestep {_f(p.dt)}\n")
    types = np.asarray(t.types)
    with open(os.path.join(dirpath, data_name), "w") as f:
        f.write("LAMMPS data file written by monomers2026_b200.casefiles\n\n")
        f.write(f"{M} atoms\n{len(t.bonds)} bonds\n{len(t.angles)} angles\n\n")
        f.write(f"{t.ntypes} atom types\n{max(1, len(t.bond_coeff) - 1)} bond types\n"
                f"{max(1, len(t.angle_coeff) - 1)} angle types\n\n")
        for ax in "xyz":
            f.write(f"{_f(p.box_lo)} {_f(p.box_hi)} {ax}lo {ax}hi\n")
        f.write("\nMasses\n\n")
        for ty in range(1, t.ntypes + 1):
            f.write(f"{ty} {_f(mass_per_type[ty])}\n")
        f.write("\nAtoms\n\n")
        for i in range(M):
            f.write(f"{i + 1} 1 {int(types[i])} {_f(x[i, 0])} {_f(x[i, 1])} {_f(x[i, 2])}\n")
        if v is not None:
            f.write("\nVelocities\n\n")
            for i in range(M):
                f.write(f"{i + 1} {_f(v[i, 0])} {_f(v[i, 1])} {_f(v[i, 2])}\n")
        if len(t.bonds):
            f.write("\nBonds\n\n")
            for b, (bt, i, j) in enumerate(np.asarray(t.bonds)):
                f.write(f"{b + 1} {bt} {i + 1} {j + 1}\n")
        if len(t.angles):
            f.write("\nAngles\n\n")
            for a, (at, i, j, k) in enumerate(np.asarray(t.angles)):
                f.write(f"{a + 1} {at} {i + 1} {j + 1} {k + 1}\n")
    return dirpath


def write_workload(dirpath: str, wl, nsteps: int | None = None) -> str:
    """Case directory of a Workload (uniform mass per type taken from the first atom of each type)."""
    t = wl.topology
    mpt = np.zeros(t.ntypes + 1)
    for ty in range(1, t.ntypes + 1):
        sel = np.nonzero(np.asarray(t.types) == ty)[0]
        mpt[ty] = wl.mass[sel[0]] if len(sel) else 1.0
    return write_case(dirpath, wl.params, wl.x, mpt, t, wl.nsteps if nsteps is None else nsteps, v=wl.v)
