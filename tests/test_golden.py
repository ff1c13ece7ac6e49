"""The oracle against golden vectors produced by the reference's own CPU code
(tests/golden/make_golden.py) on the reference's NucleotideMonomer example
case with thermal driving off: 96 four-bead molecules, harmonic bonds and
angles, lj/cut pairs (special 0 0 0), real-unit parameters, 30^3 grid."""
import os

import numpy as np
import pytest

G = os.path.join(os.path.dirname(__file__), "golden", "nucleotide_kT0.npz")


def golden():
    return np.load(G)


def golden_topology(d):
    from monomers2026_b200.selm import Topology
    return Topology(types=d["types"], ntypes=int(d["ntypes"]), bonds=d["bonds"], bond_style="harmonic",
                    bond_coeff=d["bond_coeff"], angles=d["angles"], angle_style="harmonic",
                    angle_coeff=d["angle_coeff"], pair_style="lj/cut", pair_coeff=d["pair_coeff"],
                    special_lj=(0.0, 0.0, 0.0))


def golden_params(d, form="plain64"):
    from monomers2026_b200.selm import Params
    n = d["dims"]
    return Params(numMeshPtsPerDir=(int(n[0]), int(n[1]), int(n[2])), box_lo=float(d["lo"]), box_hi=float(d["hi"]),
                  rho=float(d["rho"]), mu=float(d["mu"]), KB=float(d["KB"]), T=float(d["T"]), dt=float(d["dt"]),
                  flagStochasticDriving=0, SELM_Seed=int(d["seed"]), form=form)


def test_oracle_reproduces_reference_golden(oracle):
    d = golden()
    p = golden_params(d)
    topo = golden_topology(d).as_dict()
    mass = d["mass_per_type"][d["types"]]
    ff = oracle.ForceField(topo, p.box_lo, p.box_hi)
    o = oracle.Sim(p.numMeshPtsPerDir, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, d["x0"], mass, ff=ff)
    o.initial()
    done = 0
    for s in (1, 10, 30):
        o.step(s - done)
        done = s
        assert np.array_equal(o.x, d[f"x{s}"])
        assert np.array_equal(o.v, d[f"v{s}"])
        assert np.array_equal(o.f, d[f"f{s}"])
    assert np.array_equal(o.u.ravel()[d["u30_idx"]], d["u30_val"])


def test_golden_case_hits_the_reference_edge_weight():
    # x = 0.5 in a [-3, 3] box on 30 cells: the staggered coordinate is exactly 17.0,
    # where the reference's loop leaves the weight factor of the distance-2 point at 1.
    d = golden()
    dx = (float(d["hi"]) - float(d["lo"])) / int(d["dims"][0])
    g = (d["x0"] - float(d["lo"])) / dx - 0.5
    assert np.any(g == np.floor(g))
