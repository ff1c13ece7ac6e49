"""The CUDA path, driven through the drop-in case-directory entry point
(selm_create_from_files), against the reference's own outputs on its
NucleotideMonomer example case (tests/golden).  Tolerance: 1e-12 relative
(FP64 forms), 1e-5 (FP32 form)."""
import tempfile

import numpy as np
import pytest

from test_golden import golden, golden_params, golden_topology

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("form,tol", [("plain64", 1e-12), ("fused64", 1e-12), ("fused32", 1e-5)])
def test_case_directory_run_matches_reference(form, tol):
    import ctypes as C

    from monomers2026_b200 import _lib
    from monomers2026_b200.casefiles import write_case
    d = golden()
    p = golden_params(d, form)
    L = _lib.load()
    with tempfile.TemporaryDirectory() as tmp:
        write_case(tmp, p, d["x0"], d["mass_per_type"], golden_topology(d), 30)
        with open(tmp + "/Model.SELM", "a") as f:
            f.write(f"form {form}\n")
        h = C.c_void_p()
        _lib.check(L.selm_create_from_files(tmp.encode(), C.byref(h)))
    try:
        _lib.check(L.selm_initial(h))
        M = len(d["types"])
        dp = C.POINTER(C.c_double)
        done = 0
        for s in (1, 10, 30):
            _lib.check(L.selm_step(h, s - done))
            done = s
            x, v, f = np.zeros((M, 3)), np.zeros((M, 3)), np.zeros((M, 3))
            _lib.check(L.selm_get_particles(h, x.ctypes.data_as(dp), v.ctypes.data_as(dp), f.ctypes.data_as(dp)))
            assert rel(x, d[f"x{s}"]) < tol
            assert rel(v, d[f"v{s}"]) < tol
            assert rel(f, d[f"f{s}"]) < tol
        n = d["dims"]
        u = np.zeros(3 * int(n[0]) * int(n[1]) * int(n[2]))
        _lib.check(L.selm_get_field(h, 0, u.ctypes.data_as(dp)))
        err = np.abs(u[d["u30_idx"]] - d["u30_val"]).max() / float(d["u30_absmax"])
        assert err < tol
    finally:
        L.selm_destroy(h)
