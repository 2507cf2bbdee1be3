"""mf_solve_device_static (the device solve whose work buffers live in a fixed
device region) against mf_solve_device on the same factor.

The file name sorts last so that, in a full run, these calls come after every
other GPU test of the session; run alone, they are the first solves of a fresh
process.  Both orders must pass.
"""
import ctypes

import numpy as np
import pytest

import multifrontal as mf
from multifrontal import testmatrices as tm

pytestmark = pytest.mark.gpu

_vp, _i64 = ctypes.c_void_p, ctypes.c_int64


def _bind(lib):
    # the package binds the other entry points used here (mf_solve_device,
    # mf_synchronize, mf_last_error) with these same types
    lib.mf_solve_device_static.argtypes = [_vp, _vp, _i64, _i64, _vp]
    lib.mf_solve_device_static.restype = ctypes.c_int


def _device_block(torch, B, ldb):
    """Column-major n x k block with leading dimension ldb on cuda:0."""
    n, k = B.shape
    T = torch.zeros((k, ldb), dtype=torch.float64, device="cuda:0")
    T[:, :n] = torch.from_numpy(np.ascontiguousarray(B.T)).to("cuda:0")
    return T


@pytest.mark.parametrize("k,pad", [(4, 0), (19, 3)])
def test_static_region_solve_matches_device_solve(k, pad):
    import torch

    A = tm.grid_laplacian(60, 50, seed=21)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(60, 50, 1))
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    assert F.info == 0
    lib, h = F._handle.lib, F._handle.h
    _bind(lib)
    n, ldb = S.n, S.n + pad
    B = tm.rhs(n, k, seed=5)
    perm = torch.from_numpy(np.ascontiguousarray(P.perm, dtype=np.int64)).to("cuda:0")

    ref = _device_block(torch, B, ldb)
    torch.cuda.synchronize()
    assert lib.mf_solve_device(h, ref.data_ptr(), k, ldb, perm.data_ptr()) == 0, lib.mf_last_error()
    assert lib.mf_synchronize(h) == 0
    want = ref[:, :n].cpu().numpy().T

    # two calls in a row through the one region, each after a solve of other
    # right-hand sides (16 columns) has left different data everywhere in it
    other = _device_block(torch, tm.rhs(n, 16, seed=77), n)
    for _ in range(2):
        torch.cuda.synchronize()
        assert lib.mf_solve_device_static(h, other.data_ptr(), 16, n, perm.data_ptr()) == 0, lib.mf_last_error()
        assert lib.mf_synchronize(h) == 0
        X = _device_block(torch, B, ldb)
        torch.cuda.synchronize()
        rc = lib.mf_solve_device_static(h, X.data_ptr(), k, ldb, perm.data_ptr())
        assert rc == 0, lib.mf_last_error()
        assert lib.mf_synchronize(h) == 0
        got = X.cpu().numpy()
        np.testing.assert_allclose(got[:, :n].T, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
        assert np.all(got[:, n:] == 0.0)  # padding rows untouched
        assert tm.backward_error(A, got[:, :n].T, B).max() <= 1e-13


def test_static_region_rejects_oversize_solve():
    import torch

    A = tm.grid_laplacian(400, 400, seed=22)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(400, 400, 1))
    F = mf.ChordalCholesky(A, P, S)
    lib, h = F._handle.lib, F._handle.h
    _bind(lib)
    k = 16  # 2 * n * k alone is 5.1M doubles, above the 4,194,304 the region holds
    X = torch.zeros((k, S.n), dtype=torch.float64, device="cuda:0")
    perm = torch.from_numpy(np.ascontiguousarray(P.perm, dtype=np.int64)).to("cuda:0")
    rc = lib.mf_solve_device_static(h, X.data_ptr(), k, S.n, perm.data_ptr())
    assert rc == -1
    assert b"static region holds 4194304" in lib.mf_last_error()
