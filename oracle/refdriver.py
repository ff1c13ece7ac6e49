"""TEST INFRASTRUCTURE ONLY: the reference's own CPU code (oracle/_ref).

oracle/ref.mk compiles the reference's mpi/SELM.cpp, SELM_Eulerian_Period.cpp
and SELM_Lagrangian_LAMMPS.cpp unchanged against this project's single-rank
MPI / FFTW-MPI / LAMMPS shims.  This module runs it on a case directory.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libselm_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB)
        L.ref_create.argtypes = [C.c_char_p]
        L.ref_create.restype = C.c_void_p
        L.ref_step.argtypes = [C.c_void_p, C.c_int]
        L.ref_natoms.argtypes = [C.c_void_p]
        L.ref_dims.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
        L.ref_get.argtypes = [C.c_void_p, dp, dp, dp, dp]
        L.ref_destroy.argtypes = [C.c_void_p]
        L.ref_last_error.restype = C.c_char_p
        _lib = L
    return _lib


class ReferenceRun:
    """The reference's Selm driver (mpi/SELM.cpp) on a case directory or a workload."""

    def __init__(self, case_or_workload, nsteps: int | None = None):
        L = lib()
        if isinstance(case_or_workload, str):
            d = case_or_workload
        else:
            from monomers2026_b200.casefiles import write_workload
            self._tmp = tempfile.TemporaryDirectory()
            d = write_workload(self._tmp.name, case_or_workload, nsteps)
        h = L.ref_create(d.encode())
        if not h:
            raise RuntimeError("reference run failed to start: " + L.ref_last_error().decode())
        self.h = h
        self.M = L.ref_natoms(h)
        dims = (C.c_int * 3)()
        L.ref_dims(h, dims)
        self.dims = tuple(dims)
        self.nstep = 0

    def step(self, n: int = 1):
        lib().ref_step(self.h, n)
        self.nstep += n

    def state(self):
        nx, ny, nz = self.dims
        x = np.zeros((self.M, 3))
        v = np.zeros((self.M, 3))
        f = np.zeros((self.M, 3))
        u = np.zeros((3, nz, ny, nx))
        lib().ref_get(self.h, x, v, f, u)
        return x, v, f, u

    def close(self):
        if getattr(self, "h", None):
            lib().ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
