"""TEST AND BENCH INFRASTRUCTURE ONLY: the reference's own GPU step.

oracle/refgpu.mk compiles the reference's cuda/SELM_Eulerian_Period.cu and
cuda/SELM_Kernel.cu unchanged for sm_100a with a project-written stub driver
(oracle/refgpu_stub.cu: the Selm parameters, a Lagrangian that launches the
reference's lagrangian_update with the arguments of Lagrangian_LAMMPS::run and
holds the conservative force fixed where the reference copies LAMMPS' host
forces in, and Selm::run's step order).  It is the reference-GPU bar of the
bench and a second oracle at kT = 0 (its spreading uses FP64 atomics, so its
sums are not in a fixed order: agreement is to rounding, not bitwise).  It
also times cuFFT (R2C + C2R of three fields) as a cross-check of this
project's own FFT kernels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libselm_refgpu.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        L.refgpu_create.argtypes = [C.POINTER(C.c_int), C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp]
        L.refgpu_create.restype = C.c_void_p
        L.refgpu_step.argtypes = [C.c_void_p, C.c_int]
        L.refgpu_time.argtypes = [C.c_void_p, C.c_int, dp]
        L.refgpu_get.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.refgpu_destroy.argtypes = [C.c_void_p]
        L.refgpu_cufft_time.argtypes = [C.c_int, C.c_int, C.c_int, dp]
        _lib = L
    return _lib


class ReferenceGpuRun:
    """The reference's GPU step on a workload (its positions, velocities and
    masses); the conservative force is f0 (default zero), held fixed."""

    def __init__(self, wl, f0: np.ndarray | None = None):
        p = wl.params
        M = len(wl.mass)
        x = np.ascontiguousarray(wl.x, np.float64).reshape(M, 3)
        v = np.zeros((M, 3)) if wl.v is None else np.ascontiguousarray(wl.v, np.float64).reshape(M, 3)
        f = np.zeros((M, 3)) if f0 is None else np.ascontiguousarray(f0, np.float64).reshape(M, 3)
        m = np.ascontiguousarray(wl.mass, np.float64)
        dims = (C.c_int * 3)(*[int(d) for d in p.numMeshPtsPerDir])
        h = lib().refgpu_create(dims, p.box_lo, p.box_hi, p.dt, p.mu, p.rho, p.KB, p.T, int(p.flagStochasticDriving),
                                int(p.SELM_Seed), M, x, v, f, m)
        if not h:
            raise RuntimeError("the reference GPU step failed to start")
        self.h = h
        self.M = M
        self.dims = tuple(int(d) for d in p.numMeshPtsPerDir)

    def step(self, n: int = 1) -> None:
        if lib().refgpu_step(self.h, int(n)) != 0:
            raise RuntimeError("reference GPU step failed")

    def time(self, n: int) -> dict:
        out = np.zeros(4)
        if lib().refgpu_time(self.h, int(n), out) != 0:
            raise RuntimeError("reference GPU step failed")
        return {"lagrangian_update": out[0] / n, "fluid_update": out[1] / n, "thermal_forcing": out[2] / n,
                "step": out[3] / n}

    def state(self):
        nx, ny, nz = self.dims
        x = np.zeros((self.M, 3))
        v = np.zeros((self.M, 3))
        u = np.zeros((3, nz, ny, nx))
        if lib().refgpu_get(self.h, x.ctypes.data, v.ctypes.data, u.ctypes.data) != 0:
            raise RuntimeError("reference GPU read-back failed")
        return x, v, u

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().refgpu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cufft_time(n: int, precision: int, reps: int = 20) -> dict:
    """Mean device time (ms) of cuFFT's batched R2C and C2R of three n^3 fields."""
    out = np.zeros(2)
    rc = lib().refgpu_cufft_time(int(n), int(precision), int(reps), out)
    if rc != 0:
        raise RuntimeError(f"cuFFT timing failed ({rc})")
    return {"r2c_ms": float(out[0]), "c2r_ms": float(out[1])}
