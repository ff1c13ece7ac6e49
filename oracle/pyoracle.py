"""TEST INFRASTRUCTURE ONLY: ctypes access to the plain-C FP64 oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg load
this module; the product never does.  The C sources (selm_oracle.c) restate
the reference's step (yaohong99/monomers2026, data/src/selm-main/src/mpi and
src/cuda) and cite it line by line.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "libselm_oracle.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(dtype=np.uint32, flags="C_CONTIGUOUS")


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        L.orc_fft1.argtypes = [C.c_int, _dp, C.c_int]
        L.orc_fft3_r2c.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp]
        L.orc_fft3_c2r.argtypes = [C.c_int, C.c_int, C.c_int, _dp, _dp]
        L.orc_phi.argtypes = [C.c_double]
        L.orc_phi.restype = C.c_double
        L.orc_interp.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, C.c_int, _dp]
        L.orc_spread.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp, _dp, C.c_int]
        L.orc_fluid_run.argtypes = [_dp, _dp, _dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                    C.c_double, C.c_double]
        L.orc_noise_from_normals.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, _dp,
                                             C.c_int]
        L.orc_philox4x32.argtypes = [_u32p, _u32p, _u32p]
        L.orc_fluid_normals.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_int, _dp]
        L.orc_particle_normals.argtypes = [C.c_uint64, C.c_uint64, C.c_int, _dp]
        L.orc_lagrangian_update.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, C.c_int, C.c_int, C.c_int,
                                            C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                            C.c_double, C.c_void_p, C.c_int]
        L.orc_forces.argtypes = [C.c_void_p, _dp, _dp]
        L.orc_forces.restype = C.c_int
        L.orc_sim_initial.argtypes = [C.c_void_p]
        L.orc_sim_step.argtypes = [C.c_void_p]
        L.orc_qs_velocity.argtypes = [_dp, _dp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                      C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, C.c_uint64,
                                      C.c_uint64, _dp]
        _lib = L
    return _lib


def _c(a, dt=np.float64):
    return np.ascontiguousarray(a, dtype=dt)


# ----------------------------------------------------------------- FFT
def fft1(z: np.ndarray, sign: int) -> np.ndarray:
    z = np.ascontiguousarray(z, dtype=np.complex128).copy()
    buf = z.view(np.float64)
    lib().orc_fft1(len(z), buf, sign)
    return buf.view(np.complex128)


def rfft3(a: np.ndarray) -> np.ndarray:
    nz, ny, nx = a.shape
    out = np.zeros(nz * ny * (nx // 2 + 1) * 2)
    lib().orc_fft3_r2c(nx, ny, nz, _c(a).ravel(), out)
    return out.view(np.complex128).reshape(nz, ny, nx // 2 + 1)


def irfft3(h: np.ndarray, nx: int) -> np.ndarray:
    nz, ny, nxh = h.shape
    out = np.zeros(nz * ny * nx)
    lib().orc_fft3_c2r(nx, ny, nz, np.ascontiguousarray(h, dtype=np.complex128).view(np.float64).ravel(), out)
    return out.reshape(nz, ny, nx)


# ----------------------------------------------------------------- coupling
def phi(r: float) -> float:
    return lib().orc_phi(float(r))


def interp(u: np.ndarray, lo: float, dx: float, x: np.ndarray) -> np.ndarray:
    _, nz, ny, nx = u.shape
    x = _c(x).reshape(-1)
    M = x.size // 3
    out = np.zeros(3 * M)
    lib().orc_interp(_c(u).ravel(), nx, ny, nz, lo, dx, x, M, out)
    return out.reshape(M, 3)


def spread(fgrid: np.ndarray, lo: float, dx: float, x: np.ndarray, tf: np.ndarray) -> np.ndarray:
    _, nz, ny, nx = fgrid.shape
    g = _c(fgrid).ravel().copy()
    x = _c(x).reshape(-1)
    lib().orc_spread(g, nx, ny, nz, lo, dx, x, _c(tf).reshape(-1), x.size // 3)
    return g.reshape(3, nz, ny, nx)


def fluid_run(u: np.ndarray, fgrid: np.ndarray, dx, mu, rho, dt) -> np.ndarray:
    _, nz, ny, nx = u.shape
    out = np.zeros(u.size)
    lib().orc_fluid_run(_c(u).ravel(), out, _c(fgrid).ravel(), nx, ny, nz, dx, mu, rho, dt)
    return out.reshape(u.shape)


def qs_velocity(dims, lo, dx, x, F, mu, kB=0.0, T=0.0, dt=1.0, stochastic=False, seed=0, step=1) -> np.ndarray:
    """Quasi-steady Stokes velocity [3][Nz][Ny][Nx] of the monomer forces F (orc_qs_velocity)."""
    nx, ny, nz = dims
    x = _c(x).reshape(-1, 3)
    out = np.zeros((3, nz, ny, nx))
    lib().orc_qs_velocity(x.ravel(), _c(F).ravel(), len(x), nx, ny, nz, lo, dx, mu, kB, T, dt, int(stochastic),
                          int(seed), int(step), out.ravel())
    return out


def noise_from_normals(dims, dx, scale, xi, noise_mode=0) -> np.ndarray:
    nx, ny, nz = dims
    out = np.zeros(3 * nx * ny * nz)
    lib().orc_noise_from_normals(out, nx, ny, nz, dx, scale, _c(xi).ravel(), noise_mode)
    return out.reshape(3, nz, ny, nx)


def philox(ctr, key) -> np.ndarray:
    out = np.zeros(4, np.uint32)
    lib().orc_philox4x32(_c(ctr, np.uint32), _c(key, np.uint32), out)
    return out


def fluid_normals(seed, step, dims) -> np.ndarray:
    nx, ny, nz = dims
    n2 = (nx // 2 + 1) * ny * nz
    out = np.zeros(6 * n2)
    lib().orc_fluid_normals(seed, step, nx, ny, nz, out)
    return out.view(np.complex128).reshape(3, nz, ny, nx // 2 + 1)


def particle_normals(seed, step, M) -> np.ndarray:
    out = np.zeros(3 * M)
    lib().orc_particle_normals(seed, step, M, out)
    return out.reshape(M, 3)


# ----------------------------------------------------------------- force field
class _FF(C.Structure):
    _fields_ = [
        ("natoms", C.c_int), ("ntypes", C.c_int), ("type", C.c_void_p),
        ("nbonds", C.c_int), ("bond", C.c_void_p), ("bond_style", C.c_int), ("bond_coeff", C.c_void_p),
        ("nangles", C.c_int), ("angle", C.c_void_p), ("angle_style", C.c_int), ("angle_coeff", C.c_void_p),
        ("pair_style", C.c_int), ("pair_coeff", C.c_void_p), ("pair_shift", C.c_int),
        ("special_lj", C.c_double * 4), ("body_force", C.c_double * 3),
        ("lo", C.c_double), ("hi", C.c_double),
    ]


class ForceField:
    """Holds the arrays that back an ``orc_ff`` (keeps them alive).

    ``topo`` is a dict with keys: types (M,) 1-based, ntypes, bonds (nb,3)
    [type,i,j], bond_style ('none'|'harmonic'|'fene'), bond_coeff (ntb+1,4),
    angles (na,4) [type,i,j,k], angle_style, angle_coeff (nta+1,2),
    pair_style ('none'|'lj/cut'), pair_coeff ((nt+1)^2,3) [eps,sigma,rc],
    pair_shift, special_lj (4,), body_force (3,)."""

    BOND = {"none": 0, "harmonic": 1, "fene": 2}
    ANGLE = {"none": 0, "harmonic": 1}
    PAIR = {"none": 0, "lj/cut": 1}

    def __init__(self, topo: dict, lo: float, hi: float):
        t = topo
        self.types = _c(t["types"], np.int32)
        self.bonds = _c(t.get("bonds", np.zeros((0, 3))), np.int32).reshape(-1, 3)
        self.bond_coeff = _c(t.get("bond_coeff", np.zeros((1, 4)))).reshape(-1, 4)
        self.angles = _c(t.get("angles", np.zeros((0, 4))), np.int32).reshape(-1, 4)
        self.angle_coeff = _c(t.get("angle_coeff", np.zeros((1, 2)))).reshape(-1, 2)
        nt = int(t["ntypes"])
        self.pair_coeff = _c(t.get("pair_coeff", np.zeros(((nt + 1) ** 2, 3)))).reshape(-1, 3)
        s = _FF()
        s.natoms = len(self.types)
        s.ntypes = nt
        s.type = self.types.ctypes.data
        s.nbonds = len(self.bonds)
        s.bond = self.bonds.ctypes.data
        s.bond_style = self.BOND[t.get("bond_style", "none")]
        s.bond_coeff = self.bond_coeff.ctypes.data
        s.nangles = len(self.angles)
        s.angle = self.angles.ctypes.data
        s.angle_style = self.ANGLE[t.get("angle_style", "none")]
        s.angle_coeff = self.angle_coeff.ctypes.data
        s.pair_style = self.PAIR[t.get("pair_style", "none")]
        s.pair_coeff = self.pair_coeff.ctypes.data
        s.pair_shift = int(t.get("pair_shift", 0))
        sl = t.get("special_lj", [1.0, 0.0, 0.0, 0.0])
        for i in range(4):
            s.special_lj[i] = float(sl[i])
        bf = t.get("body_force", [0.0, 0.0, 0.0])
        for i in range(3):
            s.body_force[i] = float(bf[i])
        s.lo = lo
        s.hi = hi
        self.struct = s

    def forces(self, x: np.ndarray):
        f = np.zeros(x.size)
        warn = lib().orc_forces(C.byref(self.struct), _c(x).ravel(), f)
        return f.reshape(-1, 3), warn


# ----------------------------------------------------------------- whole step
class _Sim(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("M", C.c_int),
        ("lo", C.c_double), ("hi", C.c_double), ("dx", C.c_double), ("dt", C.c_double),
        ("mu", C.c_double), ("rho", C.c_double), ("kB", C.c_double), ("T", C.c_double),
        ("stochastic", C.c_int), ("noise_mode", C.c_int),
        ("seed", C.c_uint64), ("step", C.c_uint64),
        ("x", C.c_void_p), ("v", C.c_void_p), ("f", C.c_void_p), ("m", C.c_void_p),
        ("u", C.c_void_p), ("fgrid", C.c_void_p), ("scratch", C.c_void_p), ("ff", C.c_void_p),
        ("integrator", C.c_int),
    ]


class Sim:
    """FP64 oracle of the whole SELM step: the inertial scheme in the reference's
    driver order (integrator 0), or the project's quasi-steady form (integrator 1)."""

    def __init__(self, dims, lo, hi, dt, mu, rho, kB, T, x, m, v=None, stochastic=False, seed=0,
                 noise_mode=0, ff: ForceField | None = None, integrator=0):
        nx, ny, nz = dims
        N = nx * ny * nz
        M = len(m)
        self.dims = (nx, ny, nz)
        self.x = _c(x).reshape(M, 3).copy()
        self.v = np.zeros((M, 3)) if v is None else _c(v).reshape(M, 3).copy()
        self.f = np.zeros((M, 3))
        self.m = _c(m).copy()
        self.u = np.zeros((3, nz, ny, nx))
        self.fgrid = np.zeros((3, nz, ny, nx))
        self.scratch = np.zeros((3, nz, ny, nx))
        self.ff = ff
        s = _Sim()
        s.nx, s.ny, s.nz, s.M = nx, ny, nz, M
        s.lo, s.hi, s.dx, s.dt = lo, hi, (hi - lo) / nx, dt
        s.mu, s.rho, s.kB, s.T = mu, rho, kB, T
        s.stochastic, s.noise_mode = int(stochastic), int(noise_mode)
        s.seed, s.step = int(seed), 0
        s.x, s.v, s.f, s.m = (self.x.ctypes.data, self.v.ctypes.data, self.f.ctypes.data, self.m.ctypes.data)
        s.u, s.fgrid, s.scratch = self.u.ctypes.data, self.fgrid.ctypes.data, self.scratch.ctypes.data
        s.ff = C.addressof(ff.struct) if ff is not None else None
        s.integrator = int(integrator)
        self.s = s
        self.N = N

    def initial(self):
        lib().orc_sim_initial(C.byref(self.s))

    def step(self, n=1):
        for _ in range(n):
            lib().orc_sim_step(C.byref(self.s))

    @property
    def nstep(self):
        return self.s.step
