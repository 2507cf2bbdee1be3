"""A batch of independent matrices factored and solved as one forest on the
GPU (one grouped launch per tree level across all matrices), checked matrix
by matrix against the CPU oracle, and against the same matrix factored
alone.

Bars: plain FP64 -- solution within 1e-9 relative of the oracle's and
backward error <= 1e-13 per matrix; mixed -- backward error <= 1e-12 per
matrix (device and host measurements agree) and the solution within 1e-9
relative of the matrix solved alone."""
import numpy as np
import pytest

import multifrontal as mf
from multifrontal import batch
from multifrontal import testmatrices as tm
from oracle import oracle

pytestmark = pytest.mark.gpu


def _batch(m, seed=0, lo=6, hi=18):
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=m)
    mats = [tm.config3_matrix(int(s), seed=100 + i) for i, s in enumerate(sides)]
    orders = [mf.grid_nd_order(int(s), int(s), 1) for s in sides]
    return mats, orders


def test_batched_plain_matches_oracle_per_matrix():
    mats, orders = _batch(24, seed=1)
    B = batch.BatchedFactorization(mats, orders)
    B.factorize()
    assert B.info == 0
    rhs = [tm.rhs(A.shape[0], 4, seed=i) for i, A in enumerate(mats)]
    X = B.solve(rhs)
    for i, (A, o) in enumerate(zip(mats, orders)):
        P, S = mf.symbolic(A, alg=o)
        info, Xo, _ = oracle.factor_and_solve(A, P, S, rhs[i], 0)
        assert info == 0
        rel = np.abs(X[i] - Xo).max() / np.abs(Xo).max()
        assert rel <= 1e-9, (i, rel)
        assert tm.backward_error(A, X[i], rhs[i]).max() <= 1e-13
    B.close()


def test_batched_mixed_alone_vs_in_mix():
    mats, orders = _batch(32, seed=2)
    B = batch.BatchedFactorization(mats, orders, mixed=True)
    B.factorize()
    rhs = [tm.rhs(A.shape[0], 3, seed=50 + i) for i, A in enumerate(mats)]
    X = B.solve(rhs)
    seg = B.segment_errors()
    for i, A in enumerate(mats):
        eta = tm.backward_error(A, X[i], rhs[i]).max()
        assert eta <= 1e-12, (i, eta)
        assert abs(seg[i] - eta) <= 1e-3 * eta + 1e-16
    # the same matrices alone, each its own factorization
    for i in (0, 7, 31):
        P, S = mf.symbolic(mats[i], alg=orders[i])
        F = mf.cholesky_(mf.ChordalCholesky(mats[i], P, S, mixed=True))
        Xa = mf.ldiv(F, rhs[i])
        assert tm.backward_error(mats[i], Xa, rhs[i]).max() <= 1e-12
        assert np.abs(Xa - X[i]).max() / np.abs(Xa).max() <= 1e-9
        F.close()
    B.close()


def test_batched_failure_names_the_matrix():
    mats, orders = _batch(6, seed=4)
    A = mats[3].tolil()
    A[5, 5] = -100.0
    mats[3] = A.tocsc()
    B = batch.BatchedFactorization(mats, orders)
    with pytest.raises(mf.PosDefException):
        B.factorize()
    assert B.failed_matrix() == 3
    B.close()


def test_batched_mixed_ldlt_segments_meet_tolerance():
    """Quasidefinite KKT matrices batched as one LDLt forest, mixed form: the
    refinement runs one GMRES per (matrix, column), so every matrix reaches
    the 1e-12 bar on its own and agrees with its solution alone."""
    mats = [tm.config4(side=s, m=max(8, s ** 3 // 4), seed=20 + i) for i, s in enumerate((5, 6, 7, 6, 5))]
    orders = ["amf"] * len(mats)
    B = batch.BatchedFactorization(mats, orders, ldlt=True, mixed=True)
    B.factorize()
    rhs = [tm.rhs(A.shape[0], 2, seed=70 + i) for i, A in enumerate(mats)]
    X = B.solve(rhs)
    seg = B.segment_errors()
    for i, A in enumerate(mats):
        eta = tm.backward_error(A, X[i], rhs[i]).max()
        assert eta <= 1e-12, (i, eta)
        assert abs(seg[i] - eta) <= 1e-3 * eta + 1e-16
    for i in (0, 3):
        P, S = mf.symbolic(mats[i], alg="amf")
        F = mf.ldlt_(mf.ChordalLDLt(mats[i], P, S, mixed=True))
        Xa = mf.ldiv(F, rhs[i])
        assert tm.backward_error(mats[i], Xa, rhs[i]).max() <= 1e-12
        assert np.abs(Xa - X[i]).max() / np.abs(Xa).max() <= 1e-9
        F.close()
    B.close()
