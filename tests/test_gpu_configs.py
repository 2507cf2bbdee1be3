"""GPU parity against the CPU oracle at the benchmark configurations' own
orderings and sizes (AMF, the reference default, for configs 1, 3 and 4; the
oracle computes its own symbolic analysis and assembly), plus the drop-in
boundary entry points mf_div_impl and mf_chol_impl in the reference layout,
the row solve B / F and the device log-determinant.

Bars: factor entries within 1e-10 of the factor's largest entry (LDLt pivots
within 1e-10 of |d| + |a_kk|); solutions with backward error <= 1e-13 (plain
FP64) and within 1e-9 relative of the oracle's or 4 kappa_1 eps; mixed form
backward error <= 1e-12; log|det| within 1e-10 absolute plus 1e-12 n
relative of the oracle factor's."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import batch
from multifrontal import testmatrices as tm
from oracle import oracle

from test_gpu_parity import assert_factor_close, cond1

pytestmark = pytest.mark.gpu

_pd = ctypes.POINTER(ctypes.c_double)
_p64 = ctypes.POINTER(ctypes.c_int64)


def oracle_symbolic_matches(A, P, S):
    Po, So = oracle.symbolic(A)
    assert np.array_equal(P.perm, Po.perm)
    for f in ("resptr", "sepptr", "septgt", "reltgt", "chdptr", "chdtgt"):
        assert np.array_equal(getattr(S, f), getattr(So, f)), f
    return Po, So


def oracle_factor(A, P, S, diag):
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, diag)
    assert info == 0
    return Dval, Lval, d


def test_config1_full_size_amf():
    """Config 1 as benchmarked: 100 x 100 5-point grid, AMF, one RHS."""
    A = tm.config1(seed=1)
    P, S = mf.symbolic(A)
    Po, So = oracle_symbolic_matches(A, P, S)
    want = oracle_factor(A, Po, So, 0)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    assert_factor_close(S, F.factor_arrays(), want, 0)
    b = tm.rhs(S.n, 1, seed=5)
    X = mf.ldiv(F, b)
    assert tm.backward_error(A, X, b).max() <= 1e-13
    info, Xo, _ = oracle.factor_and_solve(A, Po, So, b, 0)
    assert np.abs(X - Xo).max() / np.abs(Xo).max() <= 1e-9
    # the mixed form on the same matrix
    Fm = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    Xm = mf.ldiv(Fm, b)
    assert tm.backward_error(A, Xm, b).max() <= 1e-12
    assert np.abs(Xm - Xo).max() / np.abs(Xo).max() <= 1e-9
    F.close(); Fm.close()


def test_config3_style_batch_amf_per_matrix():
    """Config 3 shape: 2D 9-point matrices of sides U{8..48}, weights U[0.5, 2],
    diag + 1e-3, AMF per matrix, 4 RHS, one forest; every member against its
    own oracle run (plain) and the 1e-12 bar (mixed)."""
    rng = np.random.default_rng(3)
    sides = rng.integers(8, 49, size=40)
    mats = [tm.config3_matrix(int(s), seed=1000 + i) for i, s in enumerate(sides)]
    rhs = [tm.rhs(A.shape[0], 4, seed=200 + i) for i, A in enumerate(mats)]
    for mixed in (False, True):
        Bf = batch.BatchedFactorization(mats, "amf", mixed=mixed)
        Bf.factorize()
        X = Bf.solve(rhs)
        for i, A in enumerate(mats):
            eta = tm.backward_error(A, X[i], rhs[i]).max()
            assert eta <= (1e-12 if mixed else 1e-13), (i, eta)
            if i % 5 == 0:
                Po, So = oracle.symbolic(A)
                info, Xo, _ = oracle.factor_and_solve(A, Po, So, rhs[i], 0)
                assert np.abs(X[i] - Xo).max() / np.abs(Xo).max() <= 1e-9, i
        Bf.close()


def test_config4_reduced_kkt_amf():
    """Config 4 construction at a reduced size (H = 12^3 grid + 1e-4 I, A with
    6 N(0,1) entries per row, delta = 1e-6), AMF, LDLt with static pivots,
    8 RHS: plain FP64 factor and solution against the oracle; mixed form to
    1e-12."""
    side = 12
    K = tm.config4(side=side, m=16000 * side ** 3 // 64000, seed=4)
    P, S = mf.symbolic(K)
    Po, So = oracle_symbolic_matches(K, P, S)
    want = oracle_factor(K, Po, So, 1)
    F = mf.ldlt_(mf.ChordalLDLt(K, P, S))
    assert_factor_close(S, F.factor_arrays(), want, 1, adiag=K.diagonal()[P.perm])
    B = tm.rhs(S.n, 8, seed=9)
    X = mf.ldiv(F, B)
    info, Xo, _ = oracle.factor_and_solve(K, Po, So, B, 1)
    eta, eta_o = tm.backward_error(K, X, B).max(), tm.backward_error(K, Xo, B).max()
    # the plain form is held to the oracle's own backward error on this matrix
    assert eta <= max(1e-13, 10 * eta_o), (eta, eta_o)
    rel = np.abs(X - Xo).max() / np.abs(Xo).max()
    if rel > 1e-9:
        assert rel <= 4 * cond1(K, Po, So, 1) * np.finfo(float).eps, rel
    Fm = mf.ldlt_(mf.ChordalLDLt(K, P, S, mixed=True))
    Xm = mf.ldiv(Fm, B)
    assert tm.backward_error(K, Xm, B).max() <= 1e-12
    F.close(); Fm.close()


@pytest.mark.parametrize("diag", [0, 1])
def test_div_impl_reference_layout(diag):
    """mf_chol_impl + mf_div_impl with the reference's Dval/Lval/d and B in
    elimination order (ldiv!(W, NaturalFactorization(F), B)) against the
    oracle's chol_impl!/div_impl! on the same arrays."""
    A = tm.grid_laplacian(21, 19, 5, seed=17)
    if diag:
        A = (A - 0.2 * sp.eye(A.shape[0])).tocsc()  # indefinite: static LDLt pivots
    P, S = oracle.symbolic(A)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info_o, Do, Lo, do = oracle.chol_impl(S, Dval.copy(), Lval.copy(), diag)
    assert info_o == 0
    lib = mf._native.gpulib()
    h = ctypes.c_void_p()
    p = lambda a: a.ctypes.data_as(_p64)
    assert lib.mf_create(S.n, S.nfr, p(S.resptr), p(S.sepptr), p(S.septgt), p(S.reltgt), p(S.chdptr),
                         p(S.chdtgt), p(S.Dptr), p(S.Lptr), diag, 16, 0, ctypes.byref(h)) == 0
    try:
        Dg, Lg = Dval.copy(), Lval.copy()
        dg = np.zeros(S.n)
        info = ctypes.c_int64(-1)
        assert lib.mf_chol_impl(h, Dg.ctypes.data_as(_pd), Lg.ctypes.data_as(_pd),
                                dg.ctypes.data_as(_pd) if diag else None, None, ctypes.byref(info)) == 0
        assert info.value == 0
        assert_factor_close(S, (Dg, Lg, dg), (Do, Lo, do), diag, adiag=A.diagonal()[P.perm])
        for k in (1, 5, 19):
            C = np.asfortranarray(tm.rhs(S.n, k, seed=k))
            Cg = C.copy(order="F")
            assert lib.mf_div_impl(h, Cg.ctypes.data_as(_pd), k, S.n) == 0, lib.mf_last_error()
            Co = oracle.div_impl(S, Do, Lo, do, diag, C.copy(order="F"))
            assert np.abs(Cg - Co).max() <= 1e-9 * np.abs(Co).max(), k
    finally:
        lib.mf_destroy(h)


def test_rdiv_matches_oracle():
    """B / F (rdiv!!, divide.jl:287-292) against the oracle's solve of the
    transposed system (A symmetric)."""
    A = tm.grid_laplacian(16, 16, 3, seed=5)
    P, S = mf.symbolic(A)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    B = tm.rhs(3, S.n, seed=2)
    X = mf.rdiv(B, F)
    Po, So = oracle.symbolic(A)
    info, Xo, _ = oracle.factor_and_solve(A, Po, So, np.asfortranarray(B.T), 0)
    assert np.abs(X - Xo.T).max() <= 1e-9 * np.abs(Xo).max()
    assert tm.backward_error(A, X.T, B.T).max() <= 1e-13
    F.close()


def _oracle_logabsdet(A, diag):
    P, S = oracle.symbolic(A)
    Dv, Lv, d = oracle_factor(A, P, S, diag)
    if diag:
        return float(np.sum(np.log(np.abs(d)))), float(np.prod(np.sign(d)))
    diagL = np.concatenate([np.diag(Dv[S.Dptr[j]:S.Dptr[j + 1]].reshape(S.resptr[j + 1] - S.resptr[j], -1,
                                                                       order="F"))
                            for j in range(S.nfr)])
    return float(2 * np.sum(np.log(diagL))), 1.0


@pytest.mark.parametrize("diag,indefinite", [(0, False), (1, False), (1, True)])
def test_logdet_det_on_device(diag, indefinite):
    """logabsdet / logdet / det (abstract_factorization.jl:156-179) reduced on
    the GPU against the oracle factor's diagonal."""
    A = tm.grid_laplacian(23, 22, 4, seed=71)
    if indefinite:
        A = (A - 0.37 * sp.eye(A.shape[0])).tocsc()
    cls, fac = (mf.ChordalLDLt, mf.ldlt_) if diag else (mf.ChordalCholesky, mf.cholesky_)
    P, S = mf.symbolic(A)
    F = fac(cls(A, P, S))
    la, sg = F.logabsdet()
    la_o, sg_o = _oracle_logabsdet(A, diag)
    assert sg == sg_o
    assert abs(la - la_o) <= 1e-10 + 1e-12 * S.n * abs(la_o), (la, la_o)
    if sg > 0:
        assert abs(F.logdet() - la_o) <= 1e-10 + 1e-12 * S.n * abs(la_o)
    else:
        with pytest.raises(ValueError):
            F.logdet()
    # det of a small matrix against the dense determinant
    As = tm.grid_laplacian(5, 4, seed=3)
    if indefinite:
        As = (As - 0.5 * sp.eye(As.shape[0])).tocsc()
    Ps, Ss = mf.symbolic(As)
    Fs = fac(cls(As, Ps, Ss))
    dd = np.linalg.det(As.toarray())
    assert abs(Fs.det() - dd) <= 1e-10 * abs(dd)
    if not indefinite:
        # the mixed form reports the same to single-precision accuracy
        Fm = fac(cls(A, P, S, mixed=True))
        lam, sgm = Fm.logabsdet()
        assert sgm == sg_o and abs(lam - la_o) <= 1e-4 * S.n
        Fm.close()
    F.close(); Fs.close()
