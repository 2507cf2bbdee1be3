"""Small-front factorization kernels: fronts with 16 < nj <= 32 factored one
warp per front (k_small_warp, 32-row variant; opt-in, MF_WARP_FRONT32=1)
against one CTA per front (k_small, the default; MF_WARP_FRONT32=0).  Both add
the children in the same order and apply the same update expression, so the
factors -- and the solutions -- are bitwise equal; both are checked against
the oracle (normwise backward error <= 1e-13 in FP64, <= 1e-12 refined)."""
import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

pytestmark = pytest.mark.gpu


def forest(seed):
    # 2D 9-point grids under AMF: their middle levels hold many fronts of
    # 17..32 rows, the lowest ones fronts of at most 16
    mats = [tm.config3_matrix(int(s), seed=seed + i) for i, s in enumerate([12, 19, 27, 34, 41, 16, 23, 30])]
    return sp.block_diag(mats).tocsc()


def solve_both(monkeypatch, make, B):
    X = {}
    for v in ("0", "1"):
        monkeypatch.setenv("MF_WARP_FRONT32", v)
        F = make()
        X[v] = mf.ldiv(F, B)
        F.close()
    return X


@pytest.mark.parametrize("ldlt", [False, True])
def test_warp_front32_equals_cta_front(monkeypatch, ldlt):
    A = forest(400)
    P, S = mf.symbolic(A)
    nj = S.nn() + S.na()
    assert ((nj > 16) & (nj <= 32)).sum() > 50  # the 32-row path is exercised
    B = tm.rhs(S.n, 3, seed=12)
    make = (lambda: mf.ldlt_(mf.ChordalLDLt(A, P, S))) if ldlt else (lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)))
    X = solve_both(monkeypatch, make, B)
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, int(ldlt))
    assert np.abs(X["1"] - Xo).max() <= 1e-9 * np.abs(Xo).max()


def test_warp_front32_mixed_refined(monkeypatch):
    A = forest(500)
    P, S = mf.symbolic(A)
    B = tm.rhs(S.n, 4, seed=13)
    X = solve_both(monkeypatch, lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True)), B)
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-12
