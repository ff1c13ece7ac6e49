"""CPU-side checks of the C ABI: the library loads without a GPU, exports
every entry point include/selm_b200.h declares, and the host logic rejects
bad input before touching the device."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "selm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(selm_[a-z0-9_]+)\s*\(", src)) - {"selm_force_fn"})


@pytest.fixture(scope="module")
def lib():
    from monomers2026_b200 import _lib, build
    if not os.path.exists(_lib.LIB_PATH):
        build.build()
    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    names = _declared()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), n


def test_binding_lists_match_header():
    from monomers2026_b200 import _lib
    assert sorted(_lib.EXPORTED) == _declared()


def test_version_string(lib):
    assert b"sm_100a" in lib.selm_version()


def test_create_rejects_bad_params_without_gpu(lib):
    from monomers2026_b200.selm import Params
    h = C.c_void_p()
    for bad in [dict(numMeshPtsPerDir=(32, 32, 30)), dict(numMeshPtsPerDir=(134, 134, 134)),
                dict(box_hi=-1.0), dict(dt=0.0), dict(rho=0.0)]:
        p = Params(**bad).to_c()
        assert lib.selm_create(C.byref(p), C.byref(h)) == 1  # SELM_ERR_INVALID
        assert lib.selm_last_error()


def test_operator_dims_validation(lib):
    d = (C.c_int * 3)(67, 8, 8)
    x = np.zeros(3)
    out = np.zeros(3)
    u = np.zeros(3 * 67 * 8 * 8)
    dp = C.POINTER(C.c_double)
    rc = lib.selm_op_interp(64, d, 0.0, 1.0, u.ctypes.data_as(dp), 1, x.ctypes.data_as(dp), out.ctypes.data_as(dp))
    assert rc == 1


def test_workload_generators_are_seeded():
    from monomers2026_b200 import workloads as W
    a = W.config(1)
    b = W.config(1)
    assert np.array_equal(a.x, b.x) and a.x.shape == (20, 3)
    d = np.diff(W.random_walk_chains(1, 20, 50.0, 0.0, np.random.default_rng(1)), axis=0)
    d -= 50.0 * np.round(d / 50.0)
    bl = np.linalg.norm(d, axis=1)
    np.testing.assert_allclose(bl, 1.0, rtol=1e-12)
    c2 = W.config(2, nchains=2, length=30)
    assert c2.topology.bond_style == "fene" and len(c2.topology.bonds) == 58
