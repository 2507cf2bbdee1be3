"""Levels whose largest front is very large use 512-column outer blocks
(trailing updates with K = 512).  The threshold is lowered here through
MF_WIDE_FRONT_NN, read when a handle's plan is built, so that mid-size
fronts take the wide path; the bars are those of the parity and mixed
tests: the FP64 factor within 1e-10 of the oracle's (relative to the
largest entry), solutions with backward error <= 1e-13 and within 1e-9 of
the oracle's (for the quasidefinite LDLt, whose static pivots make the
FP64 backward error depend on conditioning: factor within 1e-8, solution
within 1e-9 of the oracle's or 4 kappa_1 eps); the mixed form at backward
error <= 1e-12."""
import numpy as np
import pytest

import multifrontal as mf
from multifrontal import testmatrices as tm

from oracle import oracle
from test_gpu_parity import assert_factor_close, check_solution, cond1, oracle_factor

pytestmark = pytest.mark.gpu


@pytest.fixture
def wide(monkeypatch):
    monkeypatch.setenv("MF_WIDE_FRONT_NN", "300")


def test_wide_outer_blocks_cholesky(wide):
    A = tm.grid_laplacian(24, 24, 24, seed=5)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(24, 24, 24))
    assert max(S.nn(j) for j in range(S.nfr)) > 512
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S))
    info, want = oracle_factor(A, P, S, 0)
    assert info == 0
    assert_factor_close(S, F.factor_arrays(), want, 0)
    check_solution(A, P, S, F, tm.rhs(A.shape[0], 3, seed=2), 0)
    F.close()
    Fm = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))
    B = tm.rhs(A.shape[0], 3, seed=3)
    assert tm.backward_error(A, mf.ldiv(Fm, B), B).max() <= 1e-12
    Fm.close()


def test_wide_outer_blocks_ldlt_mixed(wide):
    A = tm.config4(side=10, m=400, seed=6)
    P, S = mf.symbolic(A, alg="mindeg")
    assert max(S.nn(j) for j in range(S.nfr)) > 512
    F = mf.ldlt_(mf.ChordalLDLt(A, P, S))
    info, want = oracle_factor(A, P, S, 1)
    assert info == 0
    assert_factor_close(S, F.factor_arrays(), want, 1, rtol=1e-8, adiag=A.diagonal()[P.perm])
    B = tm.rhs(A.shape[0], 2, seed=4)
    X = mf.ldiv(F, B)
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, 1)
    rel = np.abs(X - Xo).max() / np.abs(Xo).max()
    if rel > 1e-9:  # static pivots on a quasidefinite matrix: conditioning bound as in the parity tests
        assert rel <= 4 * cond1(A, P, S, 1) * np.finfo(float).eps, rel
    F.close()
    Fm = mf.ldlt_(mf.ChordalLDLt(A, P, S, mixed=True))
    Xm = mf.ldiv(Fm, B)
    assert tm.backward_error(A, Xm, B).max() <= 1e-12
    Fm.close()
