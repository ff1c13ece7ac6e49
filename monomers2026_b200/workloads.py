"""Seeded synthetic inputs with the shapes of the benchmark configurations.

Bead-spring chains are grown as random walks of unit steps (isotropic
directions) from a uniform-random origin in the periodic box, rejecting
steps that land closer than ``min_sep`` to an existing bead so the WCA core
starts finite (the chains of the large configuration would otherwise overlap).
Geometry seeds are ``1000 + config``; masses are 1 (the configurations give
none and the integrator needs them).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from .selm import Params, Topology

WCA_RC = 2.0 ** (1.0 / 6.0)


def random_walk_chains(nchains: int, length: int, L: float, lo: float, rng: np.random.Generator,
                       step: float = 1.0, min_sep: float = 0.0, max_tries: int = 64) -> np.ndarray:
    """Positions [nchains*length, 3] wrapped into [lo, lo+L)."""
    M = nchains * length
    x = np.zeros((M, 3))
    cell = max(min_sep, 1e-9)
    nc = max(1, int(L // cell)) if min_sep > 0 else 1
    grid: dict = {}

    def key(p):
        return tuple(((np.floor((p - lo) / L * nc)).astype(int) % nc).tolist())

    def ok(p):
        if min_sep <= 0:
            return True
        k = key(p)
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    for q in grid.get(((k[0] + dx) % nc, (k[1] + dy) % nc, (k[2] + dz) % nc), ()):
                        d = p - x[q]
                        d -= L * np.round(d / L)
                        if d @ d < min_sep * min_sep:
                            return False
        return True

    def add(i, p):
        x[i] = lo + np.mod(p - lo, L)
        if min_sep > 0:
            grid.setdefault(key(x[i]), []).append(i)

    i = 0
    for c in range(nchains):
        for attempt in range(200):
            # grow the chain; if a bead cannot be placed, drop the chain and regrow it from a new origin
            start = i
            placed = []
            while True:
                p0 = lo + rng.random(3) * L
                if ok(p0):
                    break
            add(i, p0)
            placed.append(i)
            prev = x[i].copy()
            i += 1
            stuck = False
            for _ in range(1, length):
                for t in range(max_tries):
                    d = rng.standard_normal(3)
                    d *= step / np.linalg.norm(d)
                    p = prev + d
                    if ok(lo + np.mod(p - lo, L)):
                        break
                else:
                    stuck = True
                    break
                add(i, p)
                placed.append(i)
                prev = p  # unwrapped continuation keeps bond vectors exact
                i += 1
            if not stuck:
                break
            for q in placed:
                if min_sep > 0:
                    grid[key(x[q])].remove(q)
            i = start
        else:
            raise RuntimeError("random_walk_chains: could not place a self-avoiding chain")
    return x


def chain_bonds(nchains: int, length: int, btype: int = 1) -> np.ndarray:
    b = []
    for c in range(nchains):
        o = c * length
        for k in range(length - 1):
            b.append((btype, o + k, o + k + 1))
    return np.array(b, np.int32).reshape(-1, 3)


def harmonic_chain_topology(nchains, length, K=100.0, r0=1.0, body=(0.0, 0.0, 0.0)) -> Topology:
    M = nchains * length
    return Topology(types=np.ones(M, np.int32), ntypes=1, bonds=chain_bonds(nchains, length),
                    bond_style="harmonic", bond_coeff=np.array([[0, 0, 0, 0], [K, r0, 0, 0]], float),
                    special_lj=(0.0, 0.0, 0.0), body_force=body)


def fene_wca_topology(nchains, length, K=30.0, R0=1.5, eps=1.0, sigma=1.0, body=(0.0, 0.0, 0.0)) -> Topology:
    """Kremer-Grest style: FENE bonds (with their WCA core), WCA pairs, special_bonds fene (0 1 1)."""
    M = nchains * length
    pc = np.zeros((4, 3))
    pc[1 * 2 + 1] = (eps, sigma, WCA_RC * sigma)
    return Topology(types=np.ones(M, np.int32), ntypes=1, bonds=chain_bonds(nchains, length),
                    bond_style="fene", bond_coeff=np.array([[0, 0, 0, 0], [K, R0, eps, sigma]], float),
                    pair_style="lj/cut", pair_coeff=pc, special_lj=(0.0, 1.0, 1.0), body_force=body)


@dataclass
class Workload:
    name: str
    params: Params
    x: np.ndarray
    mass: np.ndarray
    topology: Topology
    nsteps: int
    v: np.ndarray | None = None


def config(idx: int, kT: float | None = None, form: str = "plain64", body: float = 0.0, nchains: int | None = None,
           length: int | None = None, grid: int | None = None, seed: int | None = None) -> Workload:
    """Configurations 1-3 (small harmonic chain, moderate FENE, large FENE).

    ``nchains``/``length``/``grid`` shrink a configuration for parity tests."""
    rng = np.random.default_rng(1000 + idx if seed is None else seed)
    if idx == 1:
        n = grid or 32
        L = float(n)
        nc, ln = nchains or 1, length or 20
        x = random_walk_chains(nc, ln, L, 0.0, rng)
        topo = harmonic_chain_topology(nc, ln)
        p = Params(numMeshPtsPerDir=(n, n, n), box_lo=0.0, box_hi=L, rho=1.0, mu=1.0, KB=1.0,
                   T=1.0 if kT is None else kT, dt=0.01, form=form)
        steps = 1000
    elif idx in (2, 3):
        n = grid or (64 if idx == 2 else 128)
        L = float(n)
        nc = nchains or (10 if idx == 2 else 1000)
        ln = length or 100
        x = random_walk_chains(nc, ln, L, 0.0, rng, min_sep=0.95)
        topo = fene_wca_topology(nc, ln, body=(body, 0.0, 0.0))
        p = Params(numMeshPtsPerDir=(n, n, n), box_lo=0.0, box_hi=L, rho=1.0, mu=1.0, KB=1.0,
                   T=1.0 if kT is None else kT, dt=0.005, form=form)
        steps = 10000 if idx == 2 else 2000
    else:
        raise ValueError("config must be 1, 2 or 3")
    p.flagStochasticDriving = int(p.T > 0)
    p.SELM_Seed = 1000 + idx
    M = len(x)
    return Workload(name=f"config{idx}", params=p, x=x, mass=np.ones(M), topology=topo, nsteps=steps)


def fene_chain_count_for(M: int, length: int = 100) -> int:
    return max(1, int(math.ceil(M / length)))


def replica(n: int, nchains: int, length: int, kT: float, seed: int, form: str = "fused32",
            integrator: str = "inertial") -> Workload:
    """One replica of the batched ensemble: FENE + WCA chains (same force field as
    configurations 2-3) in a periodic box L = n on an n^3 grid (dx = 1), its own
    geometry and Philox seed."""
    rng = np.random.default_rng(seed)
    L = float(n)
    x = random_walk_chains(nchains, length, L, 0.0, rng, min_sep=0.95)
    topo = fene_wca_topology(nchains, length)
    p = Params(numMeshPtsPerDir=(n, n, n), box_lo=0.0, box_hi=L, rho=1.0, mu=1.0, KB=1.0, T=kT, dt=0.005,
               form=form, integrator=integrator)
    p.flagStochasticDriving = int(kT > 0)
    p.SELM_Seed = seed
    M = len(x)
    return Workload(name=f"replica{seed}", params=p, x=x, mass=np.ones(M), topology=topo, nsteps=0)


def ensemble(nrep: int = 256, grids=(32, 48, 64, 96), m_range=(50, 2000), length: int = 50,
             kT_range=(0.5, 2.0), seed: int = 1004, form: str = "fused32") -> list:
    """Configuration 4: nrep replicas, grid uniform over ``grids`` (L = N, dx = 1),
    monomer count log-uniform in ``m_range`` as chains of ``length``, kT uniform in
    ``kT_range``; replica r has geometry and Philox seed ``seed * 1000 + r``."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(nrep):
        n = int(rng.choice(grids))
        M = float(np.exp(rng.uniform(np.log(m_range[0]), np.log(m_range[1]))))
        nch = max(1, int(round(M / length)))
        kT = float(rng.uniform(*kT_range))
        out.append(replica(n, nch, length, kT, seed * 1000 + r, form=form))
    return out
