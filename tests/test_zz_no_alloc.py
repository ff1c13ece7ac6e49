"""selm_op_spread_noalloc: the spreading operator for callers that cannot let
the library allocate device memory (a host that owns the whole HBM budget
through its own pool, or one that cannot afford the device synchronisation of
cudaMalloc/cudaFree).  Its scratch is a fixed file-scope device array, so two
calls in a row must each match the allocating entry point (selm_op_spread)
on the same inputs: the second call proves that the contents left by the
first do not leak into the result.  Tolerance 1e-13 relative, as for the
other FP64 operator tests.  This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(seed, n, M):
    rng = np.random.default_rng(seed)
    lo = -2.0
    dx = 0.5
    L = n * dx
    x = lo + rng.random((M, 3)) * L
    x[0] = lo + dx * np.array([3.0, 3.5, 4.0])  # grid nodes: the distance-2 edge case
    tf = rng.standard_normal((M, 3))
    base = rng.standard_normal((3, n, n, n))
    return lo, dx, x, tf, base


def test_noalloc_spread_matches_allocating_spread_two_calls():
    import torch

    from monomers2026_b200 import _lib
    from monomers2026_b200.selm import op_spread
    L = _lib.load()
    for seed, n, M in [(1, 32, 3000), (2, 24, 500)]:
        lo, dx, x, tf, base = _case(seed, n, M)
        ref = op_spread(base, lo, dx, x, tf, 64)
        g = torch.tensor(base, dtype=torch.float64, device="cuda")
        xd = torch.tensor(x, dtype=torch.float64, device="cuda")
        td = torch.tensor(tf, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        dims = (C.c_int * 3)(n, n, n)
        rc = L.selm_op_spread_noalloc(64, dims, lo, dx, C.c_void_p(g.data_ptr()), M, C.c_void_p(xd.data_ptr()),
                                      C.c_void_p(td.data_ptr()), None)
        assert rc == 0, L.selm_last_error()
        torch.cuda.synchronize()
        got = g.cpu().numpy()
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < 1e-13


def test_noalloc_spread_rejects_sizes_beyond_its_scratch():
    import torch

    from monomers2026_b200 import _lib
    L = _lib.load()
    g = torch.zeros(3 * 8 * 8 * 8, dtype=torch.float64, device="cuda")
    x = torch.zeros(3 * 70000, dtype=torch.float64, device="cuda")
    dims = (C.c_int * 3)(8, 8, 8)
    rc = L.selm_op_spread_noalloc(64, dims, 0.0, 1.0, C.c_void_p(g.data_ptr()), 70000, C.c_void_p(x.data_ptr()),
                                  C.c_void_p(x.data_ptr()), None)
    assert rc == 1 and b"65536" in L.selm_last_error()
    big = (C.c_int * 3)(256, 256, 256)
    rc = L.selm_op_spread_noalloc(64, big, 0.0, 1.0, C.c_void_p(g.data_ptr()), 10, C.c_void_p(x.data_ptr()),
                                  C.c_void_p(x.data_ptr()), None)
    assert rc == 1 and b"4096" in L.selm_last_error()
