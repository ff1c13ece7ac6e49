"""Generates the golden vectors in this directory (run where the reference is present).

nucleotide_kT0.npz: the reference's example case selm-main/test/NucleotideMonomer
(96 four-bead molecules, 30^3 grid, LAMMPS real units), with
flagStochasticDriving set to 0, run through the reference's own CPU code
(oracle/_ref: mpi/SELM*.cpp built unchanged against single-rank shims).
Stored: the case inputs parsed from its files (so the tests need no reference
checkout) and the reference's monomer state after steps 1, 10 and 30 plus the
fluid velocity at 4000 fixed grid points after step 30.

Usage: python tests/golden/make_golden.py [reference_root]
"""
from __future__ import annotations

import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def parse_case(d):
    """Inputs of a reference case directory (the subset its files use)."""
    selm = {}
    for line in open(os.path.join(d, "Model.SELM")):
        line = line.split("#")[0].split()
        if line:
            selm[line[0]] = line[1:]
    script = [ln.split("#")[0].split() for ln in open(os.path.join(d, "Model.LAMMPS_script"))]
    script = [w for w in script if w]
    info = {"bond_coeff": {}, "angle_coeff": {}, "pair_coeff": {}}
    for w in script:
        if w[0] == "read_data":
            data = w[1]
        elif w[0] == "timestep":
            info["dt"] = float(w[1])
        elif w[0] == "bond_coeff":
            info["bond_coeff"][int(w[1])] = [float(q) for q in w[2:]]
        elif w[0] == "angle_coeff":
            info["angle_coeff"][int(w[1])] = [float(q) for q in w[2:]]
        elif w[0] == "pair_coeff":
            info["pair_coeff"][(int(w[1]), int(w[2]))] = [float(q) for q in w[3:]]
        elif w[0] == "pair_style":
            info["rc_global"] = float(w[2])
    lines = [ln.split("#")[0].split() for ln in open(os.path.join(d, data))][1:]
    sec, atoms, masses, bonds, angles = None, [], {}, [], []
    hdr = {}
    for w in lines:
        if not w:
            continue
        if w[0][0].isalpha():
            sec = w[0]
            continue
        if sec is None:
            if w[-1] == "atoms":
                hdr["natoms"] = int(w[0])
            elif w[-1] == "types" and w[1] == "atom":
                hdr["ntypes"] = int(w[0])
            elif len(w) == 4 and w[2] == "xlo":
                hdr["lo"], hdr["hi"] = float(w[0]), float(w[1])
        elif sec == "Masses":
            masses[int(w[0])] = float(w[1])
        elif sec == "Atoms":
            atoms.append((int(w[0]), int(w[2]), float(w[3]), float(w[4]), float(w[5])))
        elif sec == "Bonds":
            bonds.append((int(w[1]), int(w[2]), int(w[3])))
        elif sec == "Angles":
            angles.append((int(w[1]), int(w[2]), int(w[3]), int(w[4])))
    ids = {a[0]: i for i, a in enumerate(atoms)}
    nt = hdr["ntypes"]
    pc = np.zeros(((nt + 1) ** 2, 3))
    for (i, j), (e, s, *rc) in info["pair_coeff"].items():
        r = rc[0] if rc else info["rc_global"]
        pc[i * (nt + 1) + j] = pc[j * (nt + 1) + i] = (e, s, r)
    nbt = max(info["bond_coeff"])
    nat = max(info["angle_coeff"])
    bc = np.zeros((nbt + 1, 4))
    for t, c in info["bond_coeff"].items():
        bc[t, :len(c)] = c
    ac = np.zeros((nat + 1, 2))
    for t, c in info["angle_coeff"].items():
        ac[t] = c
    return dict(
        x0=np.array([a[2:] for a in atoms]), types=np.array([a[1] for a in atoms], np.int32),
        mass_per_type=np.array([masses.get(t, 0.0) for t in range(nt + 1)]),
        bonds=np.array([(b[0], ids[b[1]], ids[b[2]]) for b in bonds], np.int32),
        angles=np.array([(a[0], ids[a[1]], ids[a[2]], ids[a[3]]) for a in angles], np.int32),
        bond_coeff=bc, angle_coeff=ac, pair_coeff=pc, ntypes=nt, lo=hdr["lo"], hi=hdr["hi"], dt=info["dt"],
        mu=float(selm["mu"][0]), rho=float(selm["rho"][0]), KB=float(selm["KB"][0]), T=float(selm["T"][0]),
        dims=np.array([int(q) for q in selm["numMeshPtsPerDir"]]), seed=int(selm.get("SELM_Seed", ["123456"])[0]))


def main():
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SELM_REFERENCE_ROOT", "/root/reference")
    case = os.path.join(ref_root, "data/src/selm-main/test/NucleotideMonomer")
    from oracle import refdriver
    if not refdriver.available():
        raise SystemExit("build oracle/_ref first: make -f oracle/ref.mk")
    with tempfile.TemporaryDirectory() as tmp:
        for f in ("Model.SELM", "Model.LAMMPS_script", "Model.LAMMPS_read_data"):
            shutil.copy(os.path.join(case, f), tmp)
        txt = open(os.path.join(tmp, "Model.SELM")).read().replace("flagStochasticDriving 1", "flagStochasticDriving 0")
        open(os.path.join(tmp, "Model.SELM"), "w").write(txt)
        inp = parse_case(tmp)
        r = refdriver.ReferenceRun(tmp)
        out = {}
        done = 0
        for s in (1, 10, 30):
            r.step(s - done)
            done = s
            x, v, f, u = r.state()
            out[f"x{s}"], out[f"v{s}"], out[f"f{s}"] = x, v, f
        rng = np.random.default_rng(2026)
        idx = rng.choice(u.size, 4000, replace=False)
        out["u30_idx"] = idx.astype(np.int64)
        out["u30_val"] = u.ravel()[idx]
        out["u30_absmax"] = np.abs(u).max()
        r.close()
    np.savez_compressed(os.path.join(HERE, "nucleotide_kT0.npz"), **inp, **out)
    print("wrote nucleotide_kT0.npz")


if __name__ == "__main__":
    main()
