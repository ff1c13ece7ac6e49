"""Python mirror of the reference's SELM plugin surface over the C ABI.

Reference lifecycle (yaohong99/monomers2026, data/src/selm-main/src/cuda):
``Selm::Selm`` reads the parameters (SELM.cu:17-48), ``initial`` sets up the
Lagrangian and Eulerian objects (SELM.cu:55-58), ``run`` advances ``nsteps``
(SELM.cu:70-98), ``final`` releases (SELM.cu:60-63).  :class:`Selm` keeps those
names; parameters use the ``Model.SELM`` keys.  Every call goes through
``libselm_b200.so``; there is no Python compute path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import SelmParams, SelmTopology, check

FORM = {"plain64": 0, "fused64": 1, "fused32": 2}
INTEGRATOR = {"inertial": 0, "quasi_steady": 1}
NOISE = {"ref_compat": 0, "exact": 1}
BOND = {"none": 0, "harmonic": 1, "fene": 2}
ANGLE = {"none": 0, "harmonic": 1}
PAIR = {"none": 0, "lj/cut": 1}
FIELD_U, FIELD_F = 0, 1


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


@dataclass
class Params:
    """The ``Model.SELM`` keys plus box and timestep (from LAMMPS in the reference)."""
    numMeshPtsPerDir: tuple = (32, 32, 32)
    box_lo: float = 0.0
    box_hi: float = 32.0
    rho: float = 1.0
    mu: float = 1.0
    KB: float = 1.0
    T: float = 0.0
    dt: float = 0.01
    flagStochasticDriving: int = 0
    SELM_Seed: int = 123456
    form: str = "plain64"
    integrator: str = "inertial"
    noise_mode: str = "ref_compat"

    def to_c(self) -> SelmParams:
        p = SelmParams()
        for a in range(3):
            p.num_mesh_pts[a] = int(self.numMeshPtsPerDir[a])
        p.box_lo, p.box_hi = float(self.box_lo), float(self.box_hi)
        p.rho, p.mu, p.KB, p.T, p.dt = float(self.rho), float(self.mu), float(self.KB), float(self.T), float(self.dt)
        p.flag_stochastic = int(self.flagStochasticDriving)
        p.seed = int(self.SELM_Seed)
        p.form = FORM[self.form]
        p.integrator = INTEGRATOR[self.integrator]
        p.noise_mode = NOISE[self.noise_mode]
        return p


@dataclass
class Topology:
    """Force field of the LAMMPS-script subset (see include/selm_b200.h)."""
    types: np.ndarray
    ntypes: int = 1
    bonds: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    bond_style: str = "none"
    bond_coeff: np.ndarray = field(default_factory=lambda: np.zeros((1, 4)))
    angles: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    angle_style: str = "none"
    angle_coeff: np.ndarray = field(default_factory=lambda: np.zeros((1, 2)))
    pair_style: str = "none"
    pair_coeff: np.ndarray | None = None
    special_lj: tuple = (0.0, 0.0, 0.0)
    body_force: tuple = (0.0, 0.0, 0.0)

    def as_dict(self) -> dict:
        nt = self.ntypes
        pc = self.pair_coeff if self.pair_coeff is not None else np.zeros(((nt + 1) ** 2, 3))
        return dict(types=self.types, ntypes=nt, bonds=self.bonds, bond_style=self.bond_style,
                    bond_coeff=self.bond_coeff, angles=self.angles, angle_style=self.angle_style,
                    angle_coeff=self.angle_coeff, pair_style=self.pair_style, pair_coeff=pc,
                    special_lj=(1.0,) + tuple(self.special_lj), body_force=self.body_force)


class Selm:
    """One simulation: Eulerian_Period fluid + monomers, resident on the GPU."""

    def __init__(self, params: Params, x: np.ndarray, mass: np.ndarray, v: np.ndarray | None = None,
                 topology: Topology | None = None, slab: tuple[int, int] | None = None):
        """``slab=(rank, nranks)``: rank's slab of an instance decomposed over
        nranks ranks (``monomers2026_b200.decomposed``)."""
        L = _lib.load()
        self._L = L
        self.params = params
        h = C.c_void_p()
        if slab is None:
            check(L.selm_create(C.byref(params.to_c()), C.byref(h)))
        else:
            check(L.selm_slab_create(C.byref(params.to_c()), int(slab[0]), int(slab[1]), C.byref(h)))
        self._h = h
        self.M = int(len(mass))
        self._x = np.ascontiguousarray(x, np.float64).reshape(self.M, 3)
        self._m = np.ascontiguousarray(mass, np.float64)
        self._v = None if v is None else np.ascontiguousarray(v, np.float64).reshape(self.M, 3)
        check(L.selm_set_particles(h, self.M, _dp(self._x), _dp(self._v), _dp(self._m)))
        self._topo_keep = None
        self._cb_keep = None
        if topology is not None:
            self.set_topology(topology)
        n = params.numMeshPtsPerDir
        self.dims = (int(n[0]), int(n[1]), int(n[2]))

    # ------------------------------------------------------------ set-up
    def set_topology(self, t: Topology) -> None:
        nt = t.ntypes
        keep = dict(
            types=np.ascontiguousarray(t.types, np.int32),
            bonds=np.ascontiguousarray(t.bonds, np.int32).reshape(-1, 3),
            bc=np.ascontiguousarray(t.bond_coeff, np.float64).reshape(-1, 4),
            angles=np.ascontiguousarray(t.angles, np.int32).reshape(-1, 4),
            ac=np.ascontiguousarray(t.angle_coeff, np.float64).reshape(-1, 2),
            pc=np.ascontiguousarray(t.pair_coeff if t.pair_coeff is not None else np.zeros(((nt + 1) ** 2, 3)),
                                    np.float64).reshape(-1, 3),
        )
        s = SelmTopology()
        s.natoms, s.ntypes = self.M, nt
        s.type = keep["types"].ctypes.data
        s.nbonds, s.bond_style, s.nbondtypes = len(keep["bonds"]), BOND[t.bond_style], len(keep["bc"]) - 1
        s.bonds, s.bond_coeff = keep["bonds"].ctypes.data, keep["bc"].ctypes.data
        s.nangles, s.angle_style, s.nangletypes = len(keep["angles"]), ANGLE[t.angle_style], len(keep["ac"]) - 1
        s.angles, s.angle_coeff = keep["angles"].ctypes.data, keep["ac"].ctypes.data
        s.pair_style, s.pair_coeff = PAIR[t.pair_style], keep["pc"].ctypes.data
        for i in range(3):
            s.special_lj[i] = float(t.special_lj[i])
            s.body_force[i] = float(t.body_force[i])
        check(self._L.selm_set_topology(self._h, C.byref(s)))
        self._topo_keep = keep

    def set_force_callback(self, fn) -> None:
        """fn(x[M,3], v[M,3]) -> f[M,3]; plays LAMMPS' role (host round trip each step)."""
        M = self.M

        def tramp(user, natoms, x, v, f):
            try:
                xa = np.ctypeslib.as_array(x, (natoms, 3))
                va = np.ctypeslib.as_array(v, (natoms, 3))
                fa = np.ctypeslib.as_array(f, (natoms, 3))
                fa[:] = fn(xa.copy(), va.copy())
                return 0
            except Exception:  # reported as a status code by the library
                return 1

        self._cb_keep = _lib.FORCE_FN(tramp)
        check(self._L.selm_set_force_callback(self._h, self._cb_keep, None))
        del M

    # ------------------------------------------------------------ lifecycle
    def initial(self) -> None:
        check(self._L.selm_initial(self._h))

    def run(self, nsteps: int) -> None:
        check(self._L.selm_step(self._h, int(nsteps)))

    step = run

    def final(self) -> None:
        if self._h:
            b = getattr(self, "_batch", None)
            if b is not None:
                b._members.remove(self)
                self._batch = None
            self._L.selm_destroy(self._h)  # leaves its batch first
            self._h = None

    def tune(self, knob: int, value: int) -> None:
        """Set a tuning knob of the fused forms (TUNE_FFT_SPLIT, TUNE_Z_BLOCKS)."""
        check(self._L.selm_tune_set(self._h, int(knob), int(value)))

    def tuned(self, knob: int) -> int:
        v = C.c_int()
        check(self._L.selm_tune_get(self._h, int(knob), C.byref(v)))
        return int(v.value)

    def device_bytes(self) -> int:
        """Device memory this simulation holds (selm_device_bytes)."""
        n = C.c_ulonglong()
        check(self._L.selm_device_bytes(self._h, C.byref(n)))
        return int(n.value)

    def __del__(self):
        try:
            self.final()
        except Exception:
            pass

    # ------------------------------------------------------------ state
    def particles(self):
        x = np.zeros((self.M, 3))
        v = np.zeros((self.M, 3))
        f = np.zeros((self.M, 3))
        check(self._L.selm_get_particles(self._h, _dp(x), _dp(v), _dp(f)))
        return x, v, f

    def get_field(self, which: int = FIELD_U) -> np.ndarray:
        nx, ny, nz = self.dims
        out = np.zeros((3, nz, ny, nx))
        check(self._L.selm_get_field(self._h, which, _dp(out)))
        return out

    def set_field(self, which: int, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, np.float64)
        check(self._L.selm_set_field(self._h, which, _dp(a)))

    def status(self) -> int:
        w = C.c_uint()
        check(self._L.selm_status(self._h, C.byref(w)))
        return int(w.value)

    @property
    def nstep(self) -> int:
        s = C.c_ulonglong()
        check(self._L.selm_get_info(self._h, None, None, C.byref(s)))
        return int(s.value)

    # ------------------------------------------------------------ streams / timing
    def set_stream(self, stream_handle: int | None) -> None:
        check(self._L.selm_set_stream(self._h, C.c_void_p(stream_handle) if stream_handle else None))

    def synchronize(self) -> None:
        check(self._L.selm_synchronize(self._h))

    def profile(self, enable: bool) -> None:
        check(self._L.selm_profile_enable(self._h, int(enable)))

    def profile_read(self, name: str):
        ms = C.c_double()
        n = C.c_long()
        check(self._L.selm_profile_read(self._h, name.encode(), C.byref(ms), C.byref(n)))
        return float(ms.value), int(n.value)


TUNE_FFT_SPLIT = 1
TUNE_Z_BLOCKS = 2


def host_register(a: np.ndarray) -> None:
    """Page-lock a C-contiguous host array (selm_host_register) so that the
    per-step copies to and from it run as direct transfers; unregister it
    (host_unregister) before it is freed."""
    if not a.flags.c_contiguous or a.nbytes == 0:
        raise ValueError("host_register needs a non-empty C-contiguous array")
    check(_lib.load().selm_host_register(a.ctypes.data, a.nbytes))


def host_unregister(a: np.ndarray) -> None:
    check(_lib.load().selm_host_unregister(a.ctypes.data))


def tune_default(grid: int, precision: int, knob: int, value: int) -> None:
    """Value of a knob for fused-form simulations created later with this cubic
    grid size and precision (selm_tune_default)."""
    check(_lib.load().selm_tune_default(int(grid), int(precision), int(knob), int(value)))


class Batch:
    """Simulations of the fused forms stepped together by one graph launch per
    step (selm_batch_*).  Members run on the batch's stream while they belong
    to it, are stepped only through it, and give the same results bit for bit
    as when stepped alone."""

    def __init__(self, stream_handle: int | None = None):
        L = _lib.load()
        self._L = L
        h = C.c_void_p()
        check(L.selm_batch_create(C.c_void_p(stream_handle) if stream_handle else None, C.byref(h)))
        self._h = h
        self._members: list[Selm] = []

    def add(self, sim: Selm) -> None:
        check(self._L.selm_batch_add(self._h, sim._h))
        sim._batch = self
        self._members.append(sim)

    def remove(self, sim: Selm) -> None:
        check(self._L.selm_batch_remove(self._h, sim._h))
        sim._batch = None
        self._members.remove(sim)

    def run(self, nsteps: int = 1) -> None:
        check(self._L.selm_batch_step(self._h, int(nsteps)))

    step = run

    def add_job(self, sim: Selm, nsteps: int) -> None:
        """A member with a step budget (selm_batch_add_job)."""
        check(self._L.selm_batch_add_job(self._h, sim._h, int(nsteps)))
        sim._batch = self
        self._members.append(sim)

    def poll(self) -> list:
        """Jobs whose budget is spent and whose last step has finished (no wait)."""
        cap = max(1, len(self._members))
        arr = (C.c_void_p * cap)()
        n = C.c_int()
        check(self._L.selm_batch_poll(self._h, arr, cap, C.byref(n)))
        by_h = {m._h.value: m for m in self._members}
        return [by_h[arr[i]] for i in range(n.value)]

    def retire(self, sim: Selm):
        """Remove a finished job and read back its x, v, f on its own stream."""
        x = np.zeros((sim.M, 3))
        v = np.zeros((sim.M, 3))
        f = np.zeros((sim.M, 3))
        check(self._L.selm_batch_retire(self._h, sim._h, _dp(x), _dp(v), _dp(f)))
        sim._batch = None
        self._members.remove(sim)
        return x, v, f

    def __len__(self) -> int:
        return int(self._L.selm_batch_size(self._h))

    @property
    def members(self) -> list:
        return list(self._members)

    @property
    def stream(self) -> int:
        return int(self._L.selm_batch_get_stream(self._h) or 0)

    def synchronize(self) -> None:
        check(self._L.selm_batch_synchronize(self._h))

    def final(self) -> None:
        if self._h:
            for m in self._members:
                m._batch = None
            self._members = []
            self._L.selm_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.final()
        except Exception:
            pass


# ---------------------------------------------------------------- operators
def _dims(d):
    return (C.c_int * 3)(*[int(v) for v in d])


def op_interp(u: np.ndarray, lo: float, dx: float, x: np.ndarray, precision: int = 64) -> np.ndarray:
    L = _lib.load()
    _, nz, ny, nx = u.shape
    u = np.ascontiguousarray(u, np.float64)
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
    out = np.zeros_like(x)
    check(L.selm_op_interp(precision, _dims((nx, ny, nz)), lo, dx, _dp(u), len(x), _dp(x), _dp(out)))
    return out


def op_spread(fgrid: np.ndarray, lo: float, dx: float, x: np.ndarray, tf: np.ndarray,
              precision: int = 64) -> np.ndarray:
    L = _lib.load()
    _, nz, ny, nx = fgrid.shape
    g = np.ascontiguousarray(fgrid, np.float64).copy()
    x = np.ascontiguousarray(x, np.float64).reshape(-1, 3)
    tf = np.ascontiguousarray(tf, np.float64).reshape(-1, 3)
    check(L.selm_op_spread(precision, _dims((nx, ny, nz)), lo, dx, _dp(g), len(x), _dp(x), _dp(tf)))
    return g


def op_rfft3(a: np.ndarray, precision: int = 64) -> np.ndarray:
    L = _lib.load()
    nz, ny, nx = a.shape
    a = np.ascontiguousarray(a, np.float64)
    out = np.zeros(2 * nz * ny * (nx // 2 + 1))
    check(L.selm_op_fft3_r2c(precision, _dims((nx, ny, nz)), _dp(a), _dp(out)))
    return out.view(np.complex128).reshape(nz, ny, nx // 2 + 1)


def op_irfft3(h: np.ndarray, nx: int, precision: int = 64) -> np.ndarray:
    L = _lib.load()
    nz, ny, _ = h.shape
    hh = np.ascontiguousarray(h, np.complex128).view(np.float64).ravel()
    out = np.zeros((nz, ny, nx))
    check(L.selm_op_fft3_c2r(precision, _dims((nx, ny, nz)), _dp(hh), _dp(out)))
    return out
