"""kT > 0: equilibrium statistics of the GPU forms against the reference's
own CPU code (oracle/_ref, which draws its thermal forcing from RanMars
normals; the GPU forms draw Philox normals), within 3 combined standard
errors.

Chains: 24 harmonic chains of 6 monomers (K = 100, rest length 1) in a
periodic 16^3 box at kT = 1, dt = 0.01, mu = rho = 1.  Eight independent runs
on each side (own geometry seed and own noise seed per run): 500 steps to
equilibrate, then 400 samples 10 steps apart.  Per run the means of

* m<v^2>, the kinetic energy per degree of freedom (equipartition; the
  reference's explicit scheme gives about 1.27 kT at this dt, in every form),
* the bond (configurational) energy per bond,
* the static structure factor S(q) = |sum_j exp(i q.x_j)|^2 / M, averaged
  over the wavevectors of the four smallest shells 2 pi/L (1,0,0), (1,1,0),
  (1,1,1), (2,0,0) and their permutations;

the standard error of each side is the spread of its eight run means (runs
are independent; samples within a run are not).

Isolated beads: 8 monomers without bonds or pair forces in the same box,
eight independent runs of 4000 steps per side, positions unwrapped every 10
steps; the mobility is the slope of the mean squared displacement over
lags of 100 to 1000 steps divided by 6 kT (D = kT * mobility).

The runs are seeded, so the outcome is fixed for a given build: this pins
the statistics, it does not re-draw them.
"""
import numpy as np
import pytest

from monomers2026_b200 import workloads as W
from monomers2026_b200.selm import Selm
from oracle import refdriver

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not refdriver.available(), reason="oracle/_ref not built (needs the reference source)")]

RUNS, EQ, SAMPLES, EVERY = 8, 500, 400, 10
NC, LN, K, L = 24, 6, 100.0, 16.0
SHELLS = [(1, 0, 0), (1, 1, 0), (1, 1, 1), (2, 0, 0)]
NAMES = ["m<v^2>", "bond energy"] + [f"S(q) {s}" for s in SHELLS] + ["bead mobility"]


def _shell_vectors():
    out = []
    for s in SHELLS:
        vs = set()
        perms = {(s[0], s[1], s[2]), (s[0], s[2], s[1]), (s[1], s[0], s[2]), (s[1], s[2], s[0]),
                 (s[2], s[0], s[1]), (s[2], s[1], s[0])}
        for perm in perms:
            for sx in (1, -1):
                for sy in (1, -1):
                    for sz in (1, -1):
                        v = (perm[0] * sx, perm[1] * sy, perm[2] * sz)
                        if v > tuple(-c for c in v):  # one of each +-q pair (S(q) = S(-q))
                            vs.add(v)
        out.append(2 * np.pi / L * np.array(sorted(vs), float))
    return out


QV = _shell_vectors()


def _observables(x, v):
    d = x[1:] - x[:-1]
    d -= L * np.round(d / L)
    inside = np.ones(len(d), bool)
    inside[LN - 1::LN] = False  # no bond between the end of one chain and the start of the next
    r = np.sqrt((d[inside] ** 2).sum(1))
    out = [(v ** 2).mean(), (K * (r - 1.0) ** 2).mean()]
    M = len(x)
    for q in QV:
        ph = x @ q.T
        out.append(float(((np.cos(ph).sum(0) ** 2 + np.sin(ph).sum(0) ** 2) / M).mean()))
    return out


def _chains(run):
    wl = W.config(1, kT=1.0, grid=16, nchains=NC, length=LN, seed=5000 + run)
    wl.params.SELM_Seed = 7000 + run
    return wl


def _beads(run):
    wl = W.config(1, kT=1.0, grid=16, nchains=8, length=1, seed=6000 + run)
    wl.params.SELM_Seed = 8000 + run
    return wl


class _Ref:
    def __init__(self, wl, nsteps):
        self.r = refdriver.ReferenceRun(wl, nsteps=nsteps)

    def run(self, n):
        self.r.step(n)

    def xv(self):
        x, v, _, _ = self.r.state()
        return x, v

    def close(self):
        self.r.close()


class _Gpu:
    def __init__(self, wl, form):
        from dataclasses import replace
        self.s = Selm(replace(wl.params, form=form), wl.x, wl.mass, v=wl.v, topology=wl.topology)
        self.s.initial()

    def run(self, n):
        self.s.run(n)

    def xv(self):
        x, v, _ = self.s.particles()
        return x, v

    def close(self):
        assert self.s.status() == 0
        self.s.final()


def _make(side, wl, nsteps):
    return _Ref(wl, nsteps) if side == "reference" else _Gpu(wl, side)


def _chain_run_means(side, run):
    s = _make(side, _chains(run), EQ + SAMPLES * EVERY)
    s.run(EQ)
    acc = []
    for _ in range(SAMPLES):
        s.run(EVERY)
        acc.append(_observables(*s.xv()))
    s.close()
    return np.mean(acc, axis=0)


def _bead_mobility(side, run):
    wl = _beads(run)
    nst = 4000
    s = _make(side, wl, nst)
    prev, _ = s.xv()
    unwrapped = prev.copy()
    xs = [unwrapped.copy()]
    for _ in range(nst // EVERY):
        s.run(EVERY)
        x, _ = s.xv()
        dxx = x - prev
        dxx -= L * np.round(dxx / L)
        unwrapped = unwrapped + dxx
        prev = x
        xs.append(unwrapped.copy())
    s.close()
    traj = np.array(xs)  # [samples][M][3]
    lags = np.arange(10, 101, 10)  # in samples: 100 .. 1000 steps
    msd = np.array([((traj[k:] - traj[:-k]) ** 2).sum(-1).mean() for k in lags])
    t = lags * EVERY * wl.params.dt
    return np.polyfit(t, msd, 1)[0] / (6.0 * wl.params.KB * wl.params.T)


def _stats(side):
    runs = np.array([_chain_run_means(side, r) for r in range(RUNS)])
    mob = np.array([_bead_mobility(side, r) for r in range(RUNS)])
    vals = np.concatenate([runs, mob[:, None]], axis=1)
    return vals.mean(0), vals.std(0, ddof=1) / np.sqrt(RUNS)


@pytest.fixture(scope="module")
def reference_stats():
    return _stats("reference")


@pytest.mark.parametrize("form", ["fused64", "fused32", "plain64"])
def test_equilibrium_statistics_match_the_reference(reference_stats, form):
    mr, sr = reference_stats
    mg, sg = _stats(form)
    rows = []
    for name, a, b, ea, eb in zip(NAMES, mg, mr, sg, sr):
        z = (a - b) / np.hypot(ea, eb)
        rows.append(f"{name}: {a:.4f} +- {ea:.4f} vs reference {b:.4f} +- {eb:.4f} ({z:+.2f} sigma)")
    print(form, "\n  " + "\n  ".join(rows))
    for name, a, b, ea, eb in zip(NAMES, mg, mr, sg, sr):
        assert abs(a - b) < 3.0 * np.hypot(ea, eb), f"{form} {name}: {a:.4f} vs reference {b:.4f}"
