"""Selected inversion on the GPU (mf_selinv, selinv!) against the CPU
oracle's restatement of selinv.jl on the same factor pattern.

Bar: every entry of the selected inverse within 1e-10 of the largest entry
of the oracle's (both compute A^-1 on the pattern of L in FP64; the orders
of the dense operations differ)."""
import json
import os

import numpy as np
import pytest

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

from test_gpu_parity import lower_mask

pytestmark = pytest.mark.gpu

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def gpu_and_oracle(A, order="amf"):
    P, S = mf.symbolic(A, alg=order)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    mf.selinv_(F)
    Zd, Zl, _ = F.factor_arrays()
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 0)
    assert info == 0
    Wd, Wl = oracle.selinv(S, Dval, Lval)
    F.close()
    return S, (Zd, Zl), (Wd, Wl)


def assert_close(S, got, want, rtol=1e-10):
    m = lower_mask(S)
    scale = max(np.abs(want[0][m]).max(initial=0), np.abs(want[1]).max(initial=0))
    assert np.abs(got[0][m] - want[0][m]).max(initial=0) <= rtol * scale
    assert np.abs(got[1] - want[1]).max(initial=0) <= rtol * scale
    assert np.all(got[0][~m] == 0.0)  # the upper triangles of the diagonal blocks are zero


def test_selinv_known_answer():
    ka = KA["selinv"]
    A = np.array(ka["A"])
    S, got, want = gpu_and_oracle(A)
    from test_known_answers import dense_factor
    np.testing.assert_allclose(dense_factor(S, *got), np.nan_to_num(np.array(ka["Z"]), nan=0.0), atol=1e-15)


@pytest.mark.parametrize("case", ["grid2d_amf", "grid3d_nd_big_fronts", "grid3d_exact_partition"])
def test_selinv_matches_oracle(case, monkeypatch):
    if case == "grid2d_amf":
        A, order = tm.grid_laplacian(40, 37, seed=3), "amf"
    elif case == "grid3d_nd_big_fronts":
        # fronts up to nj ~ 1300: the cuBLAS path for big fronts (moderate
        # weights: the entries of A^-1 carry relative errors of order
        # kappa * eps in both computations, so a high-contrast matrix would
        # measure its conditioning, not the GPU path)
        A, order = tm.grid_laplacian(30, 30, 30, seed=5), mf.grid_nd_order(30, 30, 30)
    else:
        monkeypatch.setenv("MF_AMALGAMATE", "0")
        A, order = tm.grid_laplacian(16, 15, 14, seed=6), mf.grid_nd_order(16, 15, 14)
    S, got, want = gpu_and_oracle(A, order)
    assert_close(S, got, want)


def test_solves_refuse_after_selinv_until_refactored():
    A = tm.grid_laplacian(12, 11, seed=2)
    P, S = mf.symbolic(A)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    mf.selinv_(F)
    with pytest.raises(RuntimeError):
        mf.ldiv(F, np.ones(S.n))
    import ctypes
    x = np.ones(S.n)
    rc = F._handle.lib.mf_solve(F._handle.h, x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 1, S.n, None)
    assert rc == -1 and b"selected inverse" in F._handle.lib.mf_last_error()
    F.copyto(A)
    mf.cholesky_(F)
    b = tm.rhs(S.n, 1, seed=1)[:, 0]
    assert tm.backward_error(A, mf.ldiv(F, b), b).max() <= 1e-13
    F.close()
