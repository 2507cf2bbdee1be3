"""Mixed-precision form on the GPU: FP32 fronts (same plan, single-precision
kernels) with FP64 refinement, checked against the FP64 oracle.

Bar: normwise backward error <= 1e-12 (the refinement's default tolerance) and
the solution within 1e-9 relative of the oracle's or 4 kappa_1 eps."""
import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

from test_gpu_parity import cond1

pytestmark = pytest.mark.gpu


def check(A, P, S, F, B, diag):
    X = mf.ldiv(F, B)
    it, eta_dev = F.last_refinement
    eta = tm.backward_error(A, X, B).max()
    assert eta <= 1e-12, (eta, it)
    assert abs(eta - eta_dev) <= 1e-3 * max(eta, 1e-300) + 1e-16  # device estimate matches
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, diag)
    rel = np.abs(X - Xo).max() / np.abs(Xo).max()
    if rel > 1e-9:
        assert rel <= 4 * cond1(A, P, S, diag) * np.finfo(float).eps, rel
    return it


@pytest.mark.parametrize("case", ["grid2d", "grid3d_contrast", "grid3d_large"])
def test_mixed_cholesky(case):
    if case == "grid2d":
        A = tm.grid_laplacian(60, 50, seed=11)
        order = mf.grid_nd_order(60, 50, 1)
    elif case == "grid3d_contrast":
        A = tm.grid_laplacian(18, 17, 16, seed=12, lo=1e-3, hi=1e3, shift=1e-6)
        order = mf.grid_nd_order(18, 17, 16)
    else:
        A = tm.grid_laplacian(30, 30, 30, seed=14, lo=1e-3, hi=1e3, shift=1e-6)
        order = mf.grid_nd_order(30, 30, 30)
    P, S = mf.symbolic(A, alg=order)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    assert F.info == 0
    for k in (1, 4, 16, 19):
        it = check(A, P, S, F, tm.rhs(S.n, k, seed=k), 0)
        assert it <= 100


def test_mixed_ldlt_quasidefinite():
    K = tm.config4(side=7, m=120, per_row=6, seed=5)
    P, S = mf.symbolic(K, alg="natural")
    F = mf.ldlt_(mf.ChordalLDLt(K, P, S, mixed=True))
    assert F.info == 0
    check(K, P, S, F, tm.rhs(S.n, 8, seed=4), 1)


def test_mixed_value_refresh():
    A = tm.grid_laplacian(25, 24, 3, seed=31)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(25, 24, 3))
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    A2 = tm.grid_laplacian(25, 24, 3, seed=32)
    F.copyto(A2)
    mf.cholesky_(F)
    check(A2, P, S, F, tm.rhs(S.n, 3, seed=2), 0)


def test_mixed_not_positive_definite_reports_info():
    A = tm.grid_laplacian(30, 30, seed=3).tolil()
    A[417, 417] = -5.0
    A = A.tocsc()
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(30, 30, 1))
    F = mf.ChordalCholesky(A, P, S, mixed=True)
    with pytest.raises(mf.PosDefException):
        mf.cholesky_(F)
    assert F.used_fp64  # FP32 rejected a pivot; the FP64 factorization decided


@pytest.mark.parametrize("tensor_cores", ["1", "0"])
def test_single_precision_factor_matches_scaled_oracle(tensor_cores, monkeypatch):
    """The FP32 factor (tcgen05 3xTF32 GEMMs, or FFMA with MF_TENSOR_CORES=0)
    of S A S agrees with the FP64 oracle factor of S A S to FP32 accuracy."""
    monkeypatch.setenv("MF_TENSOR_CORES", tensor_cores)
    import scipy.sparse as sp
    from test_gpu_parity import lower_mask
    A = tm.grid_laplacian(26, 25, 24, seed=61)  # fronts up to nj ~ 1100: all tensor-core roles run
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(26, 25, 24))
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    assert not F.used_fp64
    Dg, Lg, _, sc = F.factor_arrays_mixed()
    s_orig = np.empty(S.n)
    s_orig[P.perm] = sc                      # scaling in original order
    As = sp.tril(sp.diags(s_orig) @ A @ sp.diags(s_orig)).tocsc()  # lower triangle: exact symmetry
    info, (Dw, Lw, _) = oracle_factor_scaled(As, P, S)
    m = lower_mask(S)
    scale = max(np.abs(Dw[m]).max(), np.abs(Lw).max())
    assert np.abs(Dg[m] - Dw[m]).max() <= 2e-4 * scale
    assert np.abs(Lg - Lw).max() <= 2e-4 * scale
    B = tm.rhs(S.n, 4, seed=9)
    mf.ldiv(F, B)
    it, eta = F.last_refinement
    assert eta <= 1e-12 and it <= 8, (it, eta)


def oracle_factor_scaled(As, P, S):
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, As)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 0)
    assert info == 0
    return info, (Dval, Lval, d)


def test_autotune_keeps_refined_accuracy():
    """The per-level tcgen05/FFMA choice changes only which single-precision
    kernel runs; every choice must refine to the same 1e-12 bar."""
    A = tm.grid_laplacian(24, 24, 24, seed=3)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(24, 24, 24))
    F = mf.ChordalCholesky(A, P, S, mixed=True)
    mf.cholesky_(F)
    B = tm.rhs(A.shape[0], 3, seed=1)
    X0 = mf.ldiv(F, B)
    t = F.autotune(2)
    nl = t["tc_steps"].size
    assert nl > 0 and t["tc_syrk"].size == nl
    assert set(np.unique(t["tc_steps"])) <= {0, 1}
    assert t["tuned_ms"] <= min(t["tc_ms"], t["ffma_ms"]) * 1.0001
    mf.cholesky_(F)
    X1 = mf.ldiv(F, B)
    assert tm.backward_error(A, X1, B).max() <= 1e-12
    assert np.abs(X1 - X0).max() <= 1e-9 * np.abs(X0).max()
    # FFMA tiles on every level
    F.set_kernel_choice(np.zeros(nl, np.int32), np.zeros(nl, np.int32))
    mf.cholesky_(F)
    X2 = mf.ldiv(F, B)
    assert tm.backward_error(A, X2, B).max() <= 1e-12
    assert np.abs(X2 - X0).max() <= 1e-9 * np.abs(X0).max()
    with pytest.raises(ValueError):
        F.set_kernel_choice(np.zeros(nl + 1, np.int32))
    F.close()


def _fp32_rounding_breakdown_matrix(side=12, dense=False):
    """SPD in FP64, singular once ROUNDED to FP32: unit diagonal,
    off-diagonals 1e-12 except one pair at 1 - 1e-10, which rounds to 1 in
    single precision (the pair's Schur complement 2e-10 vanishes).  No
    per-front redo can help -- the FP32 inputs have lost the information --
    so the whole factorization falls back to FP64."""
    if dense:
        n = side
        rows, cols = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
        A = sp.coo_matrix((np.ones(n * n), (rows.ravel(), cols.ravel())), shape=(n, n))
    else:
        A = tm.grid_laplacian(side, side, seed=1).tocoo()
    vals = np.where(A.row == A.col, 1.0, -1e-12)
    u, v = 40, 41  # neighbours on the grid
    vals[((A.row == u) & (A.col == v)) | ((A.row == v) & (A.col == u))] = -(1.0 - 1e-10)
    return sp.csc_matrix((vals, (A.row, A.col)), shape=A.shape)


def _fp32_cancellation_matrix(side=12, dense=False):
    """SPD with every entry exact in FP32, but a pivot that cancels to about
    1e-7 of its diagonal entry inside one front: the clique {a, b, c} with
    unit diagonal, a_ca = 0.75 and a_cb = v, the float just below
    sqrt(0.4375), so the pivot of c is 0.4375 - v^2 > 0 (exact in FP64).
    The single-precision small-pivot check flags it and the front (small:
    a separate 3-vertex component) or 64 x 64 diagonal block (dense=True:
    one 130-column front, natural order, c = column 42 in block 0) is
    factored again in FP64 from the same FP32 inputs."""
    v = np.float32(np.sqrt(0.4375))
    if float(v) ** 2 >= 0.4375:
        v = np.nextafter(v, np.float32(0))
    v = float(v)
    if dense:
        n = side
        A = np.full((n, n), -1e-12)
        np.fill_diagonal(A, 1.0)
        a, b, c = 40, 41, 42
        A[c, a] = A[a, c] = 0.75
        A[c, b] = A[b, c] = v
        return sp.csc_matrix(A)
    G = tm.grid_laplacian(side, side, seed=1).tocoo()
    G = sp.csc_matrix((np.where(G.row == G.col, 1.0, -1e-12), (G.row, G.col)), shape=G.shape)
    T = np.array([[1.0, -1e-12, 0.75], [-1e-12, 1.0, v], [0.75, v, 1.0]])
    return sp.block_diag([G, sp.csc_matrix(T)]).tocsc()


@pytest.mark.parametrize("dense", [False, True])
def test_single_precision_small_pivot_is_rescued_per_front(dense):
    """North-star precision rule: an FP32 pivot flagged by the small-pivot
    check refactors only the flagged front (nj <= 67, in the small-front
    kernel) or 64 x 64 diagonal block (blocked front) in FP64 on the GPU --
    not the whole matrix -- and the refinement still reaches 1e-12."""
    A = _fp32_cancellation_matrix(130 if dense else 12, dense=dense)
    P, S = mf.symbolic(A, alg="natural" if dense else "amf")
    if dense:
        assert S.nfr == 1 and S.n == 130
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    assert F.info == 0
    assert not F.used_fp64
    assert F.rescued >= 1
    B = tm.rhs(S.n, 3, seed=4)
    X = mf.ldiv(F, B)
    it, eta = F.last_refinement
    assert eta <= 1e-12 and tm.backward_error(A, X, B).max() <= 1e-12, (it, eta)
    # a well-conditioned matrix on the same pattern needs no rescue
    W = A.copy()
    W.data = np.where(W.data > 0.5, W.data, -1e-3)
    W.setdiag(2.0)
    F.copyto(W)
    mf.cholesky_(F)
    assert F.rescued == 0 and not F.used_fp64
    F.close()


@pytest.mark.parametrize("dense", [False, True])
def test_single_precision_rounding_breakdown_falls_back_to_fp64(dense):
    """A matrix that is singular once rounded to FP32 cannot be rescued per
    front (the FP64 redo reads the same rounded inputs): the FP32
    factorization reports it and the handle factors the matrix in FP64; the
    refined solve still meets 1e-12."""
    A = _fp32_rounding_breakdown_matrix(130 if dense else 12, dense=dense)
    P, S = mf.symbolic(A)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    assert F.info == 0
    assert F.used_fp64
    B = tm.rhs(S.n, 3, seed=4)
    X = mf.ldiv(F, B)
    it, eta = F.last_refinement
    assert eta <= 1e-12 and tm.backward_error(A, X, B).max() <= 1e-12, (it, eta)
    F.close()


def test_fp64_solves_refuse_a_stale_fp64_factor():
    """After an FP64 fallback the FP64 factor storage stays allocated; a later
    mixed factorization that stays in FP32 leaves it holding the old matrix,
    so the FP64 solves and the FP64 factor download must refuse it.  The
    fallback comes from an indefinite matrix (rejected in FP64 too)."""
    import ctypes
    A1 = tm.grid_laplacian(12, 12, seed=1).tolil()
    A1[40, 40] = -3.0
    A1 = A1.tocsc()
    A2 = tm.grid_laplacian(12, 12, seed=2)
    P, S = mf.symbolic(A1)
    F = mf.ChordalCholesky(A1, P, S, mixed=True)
    mf.cholesky_(F, check=False)
    assert F.used_fp64 and F.info != 0
    lib, h = F._handle.lib, F._handle.h
    F.copyto(A2)
    mf.cholesky_(F)
    assert not F.used_fp64 and F.info == 0
    B = tm.rhs(S.n, 2, seed=3)
    X2 = mf.ldiv(F, B)
    assert tm.backward_error(A2, X2, B).max() <= 1e-12
    Xp = np.asfortranarray(B.copy())
    rc = lib.mf_solve(h, Xp.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 2, S.n,
                      P.perm.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    assert rc == -1 and b"does not hold the current matrix" in lib.mf_last_error()
    with pytest.raises(RuntimeError):
        F.factor_arrays()
    F.close()


@pytest.mark.parametrize("ldlt", [False, True])
def test_pre_split_operands_equal_per_tile_conversion(monkeypatch, ldlt):
    """The tensor-core trailing updates and SYRK reading operands split into
    TF32 hi / lo once (k_tc_split, MF_TC_SPLIT=1, the default) compute the
    same products in the same order as the kernels converting per tile
    (MF_TC_SPLIT=0): the single-precision factors are bitwise equal."""
    if ldlt:
        A = tm.config4(side=12, m=432, per_row=6, seed=9)  # a 633-column front: trailing updates
        P, S = mf.symbolic(A)
    else:
        A = tm.grid_laplacian(30, 29, 28, seed=17, lo=1e-2, hi=1e2)
        P, S = mf.symbolic(A, alg=mf.grid_nd_order(30, 29, 28))
    out = {}
    for v in ("0", "1"):
        monkeypatch.setenv("MF_TC_SPLIT", v)
        F = (mf.ldlt_ if ldlt else mf.cholesky_)((mf.ChordalLDLt if ldlt else mf.ChordalCholesky)(A, P, S, mixed=True))
        assert F.info == 0 and not F.used_fp64
        out[v] = F.factor_arrays_mixed()
        B = tm.rhs(S.n, 2, seed=3)
        X = mf.ldiv(F, B)
        assert tm.backward_error(A, X, B).max() <= 1e-12
        F.close()
    for a, b in zip(out["0"], out["1"]):
        assert np.array_equal(a, b)
