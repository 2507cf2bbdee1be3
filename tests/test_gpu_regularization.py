"""DynamicRegularization on the GPU (mf_set_regularization + mf_factorize)
against the CPU oracle's restatement of the reference's regularized
factorization (the generic recursive potrf! with regularize(), potrf.jl:3-41
and :135-178, dynamic_regularization.jl:75-90).

Bars as the parity tests: factor entries within 1e-10 of the factor's
largest entry; LDLt pivots within 1e-10 of their error scale."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

from test_gpu_parity import assert_factor_close

pytestmark = pytest.mark.gpu

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))


def test_dynamic_regularization_known_answer():
    ka = KA["dynamic_regularization"]
    A = np.array(ka["A"])
    P, S = mf.symbolic(A)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S), reg=mf.DynamicRegularization())
    assert F.info == 0
    from test_known_answers import dense_factor
    Dv, Lv, _ = F.factor_arrays()
    L = dense_factor(S, Dv, Lv)
    np.testing.assert_allclose((L @ L.T)[np.ix_(P.invp, P.invp)], np.array(ka["B"]), rtol=5e-6)
    # without the regularization the same matrix is not positive definite
    F.copyto(A)
    with pytest.raises(mf.PosDefException):
        mf.cholesky_(F)


def _negative_root_pivots(A, P, S):
    """A with the diagonal of the last column of every elimination-tree root
    lowered by 1.5 times that column's pivot, so exactly those pivots come out
    negative and are regularized; no later pivot depends on them (a pivot
    replaced by delta earlier in the tree would grow every later Schur
    complement by 1/delta and overflow on a deep tree)."""
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dw, _, _ = oracle.chol_impl(S, Dval, Lval, 0)
    assert info == 0
    A = A.tolil()
    for j in S.roots():
        nn = S.nn(j)
        c = S.res(j)[-1]
        piv = Dw[S.Dptr[j] + (nn - 1) * (nn + 1)] ** 2
        v = P.perm[c]
        A[v, v] = A[v, v] - 1.5 * piv
    return A.tocsc()


@pytest.mark.parametrize("big", [False, True])
def test_dynamic_regularization_matches_oracle(big):
    """Negative pivots at the roots' last columns are replaced by delta on the
    GPU exactly as in the oracle; small fronts (k_small: nine separate 7 x 6
    grids, nine roots) and a blocked front (k_diag: the 3D grid's root)."""
    if big:
        A = tm.grid_laplacian(26, 25, 24, seed=8)
        order = mf.grid_nd_order(26, 25, 24)
    else:
        A = sp.block_diag([tm.grid_laplacian(7, 6, seed=8 + i) for i in range(9)]).tocsc()
        order = "amf"
    P, S = mf.symbolic(A, alg=order)
    A = _negative_root_pivots(A, P, S)
    with pytest.raises(mf.PosDefException):
        mf.cholesky_(mf.ChordalCholesky(A, P, S))
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S), reg=mf.DynamicRegularization())
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dw, Lw, dw = oracle.chol_impl(S, Dval, Lval, 0, reg=(-1.0, -1.0))
    assert info == 0 and F.info == 0
    assert np.all(np.isfinite(Dw)) and np.all(np.isfinite(Lw))
    assert_factor_close(S, F.factor_arrays(), (Dw, Lw, dw), 0, rtol=1e-9)
    F.close()


def test_dynamic_regularization_ldlt_with_signs():
    """Quasidefinite KKT matrix with the pivot signs (+1 on H, -1 on the
    constraint block) and a tiny delta: pivots of the wrong sign are
    replaced by delta * s; GPU and oracle agree."""
    K = tm.config4(side=7, m=120, seed=5)
    n = K.shape[0]
    signs = np.where(np.arange(n) < 343, 1.0, -1.0)
    P, S = mf.symbolic(K)
    F = mf.ldlt_(mf.ChordalLDLt(K, P, S), signs=signs, reg=mf.DynamicRegularization())
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, K)
    info, Dw, Lw, dw = oracle.chol_impl(S, Dval, Lval, 1, signs=signs[P.perm], reg=(-1.0, -1.0))
    assert info == 0 and F.info == 0
    assert_factor_close(S, F.factor_arrays(), (Dw, Lw, dw), 1, adiag=K.diagonal()[P.perm])
    F.close()
