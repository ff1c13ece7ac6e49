"""selm_op_spread_noalloc: the spreading operator for callers that cannot let
the library allocate device memory (a host that owns the whole HBM budget
through its own pool, or one that cannot afford the device synchronisation of
cudaMalloc/cudaFree).  Its scratch is a fixed file-scope device array that
every call shares, so the test makes several calls in a row and checks each
against the allocating entry point (selm_op_spread) on the same inputs:

* FP64 (tolerance 1e-13 relative, as for the other FP64 operator tests) and
  FP32 (1e-6 relative; both entry points run the same FP32 kernels);
* on the legacy default stream and on a torch side stream;
* a small case after a larger one, repeated, must give the same grid bit for
  bit: counts and tile lists left in the array by the larger call must not
  leak into the result.

This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = {64: 1e-13, 32: 1e-6}


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


def _noalloc(L, prec, n, lo, dx, x, tf, base, stream):
    import torch
    dt = torch.float64 if prec == 64 else torch.float32
    g = torch.tensor(base, dtype=dt, device="cuda")
    xd = torch.tensor(x, dtype=torch.float64, device="cuda")
    td = torch.tensor(tf, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    dims = (C.c_int * 3)(n, n, n)
    sp = None if stream is None else C.c_void_p(stream.cuda_stream)
    rc = L.selm_op_spread_noalloc(prec, dims, lo, dx, C.c_void_p(g.data_ptr()), len(x), C.c_void_p(xd.data_ptr()),
                                  C.c_void_p(td.data_ptr()), sp)
    assert rc == 0, L.selm_last_error()
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return g.double().cpu().numpy()


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("side_stream", [False, True])
def test_noalloc_spread_matches_allocating_spread_calls_in_a_row(prec, side_stream):
    import torch

    from monomers2026_b200 import _lib
    from monomers2026_b200.selm import op_spread
    L = _lib.load()
    stream = torch.cuda.Stream() if side_stream else None
    small = None
    for seed, n, M in [(2, 24, 500), (1, 32, 3000), (2, 24, 500)]:
        lo, dx, x, tf, base = _case(seed, n, M)
        base_in = base if prec == 64 else base.astype(np.float32).astype(np.float64)
        ref = op_spread(base_in, lo, dx, x, tf, prec)
        got = _noalloc(L, prec, n, lo, dx, x, tf, base_in, stream)
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err < TOL[prec], f"n={n} M={M}: rel err {err:.3e}"
        if n == 24:
            if small is None:
                small = got
            else:
                assert np.array_equal(got, small)


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
    # 256 x 256 x 128 cells: 16 * 32 * 8 = 4096 tiles fit; 256^3 needs 8192
    big = (C.c_int * 3)(256, 256, 256)
    rc = L.selm_op_spread_noalloc(64, big, 0.0, 1.0, C.c_void_p(g.data_ptr()), 10, C.c_void_p(x.data_ptr()),
                                  C.c_void_p(x.data_ptr()), None)
    assert rc == 1 and b"4096" in L.selm_last_error()
