"""GPU numeric phase (libmfgpu.so, through the C ABI) against the CPU oracle
on the same seeded inputs.

Bars (stated per test): the factor entries agree with the oracle to
rtol 1e-10 relative to each front's largest entry; solutions have normwise
backward error <= 1e-13 and agree with the oracle's to 1e-9 relative.
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

pytestmark = pytest.mark.gpu

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))
CHOL_ORDER = np.array([3, 1, 4, 2, 5]) - 1


def lower_mask(S):
    """Boolean mask over Dval selecting the lower triangle of each block."""
    m = np.zeros(S.ndz, bool)
    for j in range(S.nfr):
        nn = S.nn(j)
        r, c = np.indices((nn, nn))
        m[S.Dptr[j]:S.Dptr[j] + nn * nn] = (r >= c).ravel(order="F")
    return m


def diag_mask(S):
    m = np.zeros(S.ndz, bool)
    for j in range(S.nfr):
        nn = S.nn(j)
        m[S.Dptr[j] + np.arange(nn) * (nn + 1)] = True
    return m


def ldlt_pivot_scale(S, Dval, Lval, d, adiag):
    """|a_kk| + sum_j L_kj^2 |d_j|: the scale of the rounding error of the
    pivot d_k = a_kk - sum_j L_kj^2 d_j (the standard LDLt error bound
    |L D L^T - A| <= gamma (|A| + |L| |D| |L^T|)); on quasidefinite matrices
    with tiny static pivots the terms can exceed |d_k| + |a_kk| by 1e6."""
    sc = np.abs(np.asarray(adiag, float)).copy()
    for j in range(S.nfr):
        r0, r1 = S.resptr[j], S.resptr[j + 1]
        nn, na = r1 - r0, S.sepptr[j + 1] - S.sepptr[j]
        D = Dval[S.Dptr[j]:S.Dptr[j] + nn * nn].reshape(nn, nn, order="F")
        L = Lval[S.Lptr[j]:S.Lptr[j] + nn * na].reshape(na, nn, order="F")
        dj = np.abs(d[r0:r1])
        sc[r0:r1] += (np.tril(D, -1) ** 2) @ dj
        sc[S.sep(j)] += (L ** 2) @ dj
    return sc


def assert_factor_close(S, got, want, diag, rtol=1e-10, adiag=None):
    """Factor entries within rtol of each factor's largest entry; LDLt pivots
    within rtol of |d| + |a_kk| + sum_j L_kj^2 |d_j| (a pivot is a_kk minus
    a sum of terms of that size, so cancellation leaves an absolute error on
    that scale; see ldlt_pivot_scale)."""
    Dg, Lg, dg = got
    Dw, Lw, dw = want
    m = lower_mask(S)
    if diag:
        m &= ~diag_mask(S)  # LDLt: unit diagonal implied, stored value unspecified
    scale = max(np.abs(Dw[m]).max(initial=0), np.abs(Lw).max(initial=0), 1e-300)
    np.testing.assert_allclose(Dg[m], Dw[m], rtol=0, atol=rtol * scale)
    np.testing.assert_allclose(Lg, Lw, rtol=0, atol=rtol * scale)
    if diag:
        scale = np.abs(dw[:S.n]) + ldlt_pivot_scale(S, Dw, Lw, dw, np.zeros(S.n) if adiag is None else adiag)
        assert np.all(np.abs(dg - dw[:S.n]) <= rtol * scale), np.max(np.abs(dg - dw[:S.n]) / scale)


def oracle_factor(A, P, S, diag, signs=None):
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    sg = None if signs is None else np.asarray(signs, float)[P.perm]
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, diag, signs=sg)
    return info, (Dval, Lval, d)


def cond1(A, P, S, diag):
    """1-norm condition estimate kappa_1(A) = ||A||_1 ||A^-1||_1 with the
    Hager/Higham estimator (the reference's condest1, operator.jl:348),
    A^-1 applied through the oracle factorization."""
    import scipy.sparse.linalg as sla
    n = S.n
    def solve(b):
        info, x, _ = oracle.factor_and_solve(A, P, S, np.asarray(b, float).reshape(n, -1), diag)
        return x
    op = sla.LinearOperator((n, n), matvec=lambda v: solve(v)[:, 0], rmatvec=lambda v: solve(v)[:, 0],
                            matmat=solve, rmatmat=solve, dtype=float)
    return float(abs(A).sum(axis=0).max()) * float(sla.onenormest(op))


def check_solution(A, P, S, F, B, diag):
    """Backward error <= 1e-13; the solution agrees with the oracle's to
    1e-9 relative, or to 4 kappa_1 eps where the problem's conditioning
    makes 1e-9 unattainable for two backward-stable solvers."""
    X = mf.ldiv(F, B)
    eta = tm.backward_error(A, X, B)
    assert eta.max() <= 1e-13, eta.max()
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, diag)
    assert info == 0
    rel = np.abs(X - Xo).max() / np.abs(Xo).max()
    if rel > 1e-9:
        kappa = cond1(A, P, S, diag)
        assert rel <= 4 * kappa * np.finfo(float).eps, (rel, kappa)
    return X


def test_known_answer_cholesky():
    ka = KA["cholesky"]
    A = np.array(ka["A"])
    P, S = mf.symbolic(A, alg=CHOL_ORDER)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    assert mf.issuccess(F)
    Dval, Lval, _ = F.factor_arrays()
    from test_known_answers import dense_factor
    np.testing.assert_allclose(dense_factor(S, Dval, Lval), np.nan_to_num(np.array(ka["L"])), atol=1e-15)
    np.testing.assert_allclose(mf.ldiv(F, np.array(ka["b"])), np.array(ka["x"]), atol=1e-15)
    assert abs(F.logdet() - np.log(np.linalg.det(A))) < 1e-12


@pytest.mark.parametrize("use_signs", [False, True])
def test_known_answer_ldlt(use_signs):
    ka = KA["ldlt"]
    A = np.array(ka["A"])
    P, S = mf.symbolic(A, alg=CHOL_ORDER)
    F = mf.ldlt_(mf.ChordalLDLt(A, P, S), signs=np.array(ka["signs"]) if use_signs else None)
    Dval, Lval, d = F.factor_arrays()
    np.testing.assert_allclose(d, np.array(ka["d_signs" if use_signs else "d"]), atol=1e-15)
    np.testing.assert_allclose(mf.ldiv(F, np.array(ka["b"])), np.array(ka["x"]), atol=1e-15)


@pytest.mark.parametrize("case", ["grid2d", "grid3d", "grid2d9", "grid3d_large"])
def test_cholesky_parity(case):
    if case == "grid2d":
        A = tm.grid_laplacian(60, 50, seed=11)
        order = mf.grid_nd_order(60, 50, 1)
    elif case == "grid3d":
        A = tm.grid_laplacian(18, 17, 16, seed=12, lo=1e-3, hi=1e3, shift=1e-6)
        order = mf.grid_nd_order(18, 17, 16)
    elif case == "grid2d9":
        A = tm.grid_laplacian(40, 40, stencil=9, seed=13, lo=0.5, hi=2.0, dist="uniform", shift=1e-3)
        order = mf.grid_nd_order(40, 40, 1)
    else:
        # fronts up to nj ~ 1300: every blocked kernel runs in several waves
        A = tm.grid_laplacian(30, 30, 30, seed=14, lo=1e-3, hi=1e3, shift=1e-6)
        order = mf.grid_nd_order(30, 30, 30)
    P, S = mf.symbolic(A, alg=order)
    info, want = oracle_factor(A, P, S, 0)
    assert info == 0
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    assert F.info == 0
    assert_factor_close(S, F.factor_arrays(), want, 0)
    for k in (1, 4, 16, 19):
        check_solution(A, P, S, F, tm.rhs(S.n, k, seed=k), 0)
    # a vector right-hand side takes the same path
    b = tm.rhs(S.n, 1, seed=99)[:, 0]
    x = mf.ldiv(F, b)
    assert x.shape == b.shape


def test_ldlt_quasidefinite_parity():
    K = tm.config4(side=7, m=120, per_row=6, seed=5)
    P, S = mf.symbolic(K, alg="natural")
    info, want = oracle_factor(K, P, S, 1)
    assert info == 0
    F = mf.ldlt_(mf.ChordalLDLt(K, P, S))
    assert_factor_close(S, F.factor_arrays(), want, 1, adiag=K.diagonal()[P.perm])
    B = tm.rhs(S.n, 8, seed=4)
    X = mf.ldiv(F, B)
    info, Xo, _ = oracle.factor_and_solve(K, P, S, B, 1)
    assert np.abs(X - Xo).max() / np.abs(Xo).max() <= 1e-9
    assert tm.backward_error(K, X, B).max() <= 1e-12


def test_ldlt_blocked_fronts_parity():
    # 3D grid shifted to be indefinite: LDLt with static pivots, big fronts
    A = tm.grid_laplacian(14, 13, 12, seed=21)
    A = (A - 0.3 * sp.eye(A.shape[0])).tocsc()
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(14, 13, 12))
    info, want = oracle_factor(A, P, S, 1)
    assert info == 0
    F = mf.ldlt_(mf.ChordalLDLt(A, P, S))
    assert_factor_close(S, F.factor_arrays(), want, 1, rtol=1e-8, adiag=A.diagonal()[P.perm])
    B = tm.rhs(S.n, 3, seed=5)
    X = mf.ldiv(F, B)
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, 1)
    assert np.abs(X - Xo).max() / np.abs(Xo).max() <= 1e-8


def test_not_positive_definite_reports_reference_info():
    A = tm.grid_laplacian(30, 30, seed=3)
    A = A.tolil()
    A[417, 417] = -5.0
    A = A.tocsc()
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(30, 30, 1))
    info_o, _ = oracle_factor(A, P, S, 0)
    assert info_o > 0
    F = mf.ChordalCholesky(A, P, S)
    with pytest.raises(mf.PosDefException) as ei:
        mf.cholesky_(F)
    assert ei.value.info == P.perm[info_o - 1] + 1
    F2 = mf.cholesky_(mf.ChordalCholesky(A, P, S), check=False)
    assert not mf.issuccess(F2)


@pytest.mark.parametrize("amalgamate", ["0", "1"])
def test_exact_and_amalgamated_partitions_agree(amalgamate, monkeypatch):
    """The device plan may merge reference fronts; the reference-layout
    factor must not depend on it."""
    monkeypatch.setenv("MF_AMALGAMATE", amalgamate)
    A = tm.grid_laplacian(22, 21, 20, seed=51, lo=1e-3, hi=1e3, shift=1e-6)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(22, 21, 20))
    info, want = oracle_factor(A, P, S, 0)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    assert_factor_close(S, F.factor_arrays(), want, 0)
    check_solution(A, P, S, F, tm.rhs(S.n, 4, seed=8), 0)
    Fl = mf.ldlt_(mf.ChordalLDLt(A, P, S))
    info, wantl = oracle_factor(A, P, S, 1)
    assert_factor_close(S, Fl.factor_arrays(), wantl, 1, adiag=A.diagonal()[P.perm])


def test_value_refresh_on_cached_pattern():
    A = tm.grid_laplacian(25, 24, 3, seed=31)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(25, 24, 3))
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    A2 = tm.grid_laplacian(25, 24, 3, seed=32)
    F.copyto(A2)
    mf.cholesky_(F)
    info, want = oracle_factor(A2, P, S, 0)
    assert_factor_close(S, F.factor_arrays(), want, 0)
    check_solution(A2, P, S, F, tm.rhs(S.n, 2, seed=1), 0)


def test_reference_layout_boundary():
    """mf_chol_impl takes and returns the reference's Dval/Lval arrays."""
    A = tm.grid_laplacian(20, 20, 4, seed=41)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(20, 20, 4))
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dg, Lg, d = mf.chol_impl(S, Dval.copy(), Lval.copy(), diag=0)
    assert info == 0
    info_o, want = oracle_factor(A, P, S, 0)
    assert_factor_close(S, (Dg, Lg, d), want, 0)


def test_rdiv_row_rhs():
    A = tm.grid_laplacian(16, 16, seed=5)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(16, 16, 1))
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    B = tm.rhs(3, S.n, seed=2)
    X = mf.rdiv(B, F)
    np.testing.assert_allclose(X @ A, B, atol=1e-10)
