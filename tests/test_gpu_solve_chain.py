"""The blocked fronts' super-block solve chain as one persistent k_s_chain
launch per level and direction (MF_SOLVE_CHAIN=1; by default only levels
of 64 or more steps) against the per-step launches (MF_SOLVE_CHAIN=0), the
small-front subtrees in one launch per direction (MF_SUBTREE_SOLVE=1)
against the per-level launches, the single-super-block levels as one
cluster launch per level and direction (MF_MID_SOLVE=1) against the
per-kernel launches, and fronts of at most 16 rows solved 16 lanes each
(MF_TINY_SOLVE=1, the default) against one warp each: the items do the same
arithmetic in the same order, so the solutions must be bitwise equal; all
are checked against the oracle (normwise backward error <= 1e-13, FP64;
<= 1e-12 refined)."""
import numpy as np
import pytest

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

pytestmark = pytest.mark.gpu


def grid(nx, ny, nz, seed):
    A = tm.grid_laplacian(nx, ny, nz, seed=seed, lo=1e-2, hi=1e2)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(nx, ny, nz))
    return A, P, S


def both(monkeypatch, make, B, var="MF_SOLVE_CHAIN"):
    X = {}
    for v in ("0", "1"):
        monkeypatch.setenv(var, v)
        F = make()
        X[v] = mf.ldiv(F, B)
        F.close()
    return X


@pytest.mark.parametrize("ldlt", [False, True])
@pytest.mark.parametrize("nrhs", [1, 3, 16])
def test_chain_equals_per_step_launches(monkeypatch, ldlt, nrhs):
    # root separator 32 x 30 = 960 columns (4 super-blocks), two 480-column
    # fronts on the level below it: several fronts per level with 2-4 steps
    A, P, S = grid(32, 30, 31, seed=61)
    B = tm.rhs(S.n, nrhs, seed=nrhs)
    make = (lambda: mf.ldlt_(mf.ChordalLDLt(A, P, S))) if ldlt else (lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)))
    X = both(monkeypatch, make, B)
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, int(ldlt))
    assert np.abs(X["1"] - Xo).max() <= 1e-9 * np.abs(Xo).max()


def test_chain_mixed_refined(monkeypatch):
    A, P, S = grid(30, 29, 28, seed=62)
    B = tm.rhs(S.n, 4, seed=3)
    X = both(monkeypatch, lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True)), B)
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-12


def test_chain_partial_last_super_block(monkeypatch):
    # a root of 21 x 19 = 399 columns: one full super-block and a 143-column one
    A, P, S = grid(21, 19, 24, seed=63)
    B = tm.rhs(S.n, 2, seed=4)
    X = both(monkeypatch, lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)), B)
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13


@pytest.mark.parametrize("ldlt", [False, True])
def test_subtree_solves_equal_per_level_launches(monkeypatch, ldlt):
    """Small fronts as subtree tasks (own update-block regions, one CTA per
    task) give the per-level results bit for bit: a 2D grid under AMF (most
    fronts small) and a batch-like forest of separate grids."""
    import scipy.sparse as sp
    A = sp.block_diag([tm.grid_laplacian(40, 38, seed=64)] + [tm.grid_laplacian(9, 8, seed=70 + i) for i in range(12)]).tocsc()
    P, S = mf.symbolic(A)
    B = tm.rhs(S.n, 3, seed=5)
    make = (lambda: mf.ldlt_(mf.ChordalLDLt(A, P, S))) if ldlt else (lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)))
    X = both(monkeypatch, make, B, var="MF_SUBTREE_SOLVE")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13


@pytest.mark.parametrize("ldlt", [False, True])
@pytest.mark.parametrize("nrhs", [1, 3, 16])
def test_mid_levels_equal_per_kernel_launches(monkeypatch, ldlt, nrhs):
    """A 3D grid under geometric nested dissection: most levels hold only
    single-super-block fronts (one cluster launch per level and direction),
    the top levels keep the stepped kernels."""
    A, P, S = grid(20, 19, 18, seed=65)
    B = tm.rhs(S.n, nrhs, seed=6 + nrhs)
    make = (lambda: mf.ldlt_(mf.ChordalLDLt(A, P, S))) if ldlt else (lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)))
    X = both(monkeypatch, make, B, var="MF_MID_SOLVE")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, int(ldlt))
    assert np.abs(X["1"] - Xo).max() <= 1e-9 * np.abs(Xo).max()


@pytest.mark.parametrize("ldlt", [False, True])
def test_mid_levels_mixed_refined(monkeypatch, ldlt):
    A, P, S = grid(24, 23, 22, seed=66)
    B = tm.rhs(S.n, 4, seed=8)
    make = ((lambda: mf.ldlt_(mf.ChordalLDLt(A, P, S, mixed=True))) if ldlt
            else (lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True))))
    X = both(monkeypatch, make, B, var="MF_MID_SOLVE")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-12


def test_mid_level_root_without_l21(monkeypatch):
    """An 8 x 8 x 8 grid: the root front (a 64-column separator, no L21) is
    itself a single-super-block level, and the 2D 60 x 50 grid under AMF
    adds levels that mix warp-per-front fronts with cluster fronts."""
    import scipy.sparse as sp
    A = sp.block_diag([tm.grid_laplacian(8, 8, 8, seed=67), tm.grid_laplacian(60, 50, seed=68)]).tocsc()
    P, S = mf.symbolic(A)
    B = tm.rhs(S.n, 2, seed=9)
    X = both(monkeypatch, lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)), B, var="MF_MID_SOLVE")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13


@pytest.mark.parametrize("ldlt", [False, True])
@pytest.mark.parametrize("nrhs", [1, 4, 16])
def test_tiny_fronts_equal_warp_per_front(monkeypatch, ldlt, nrhs):
    """Fronts with at most 16 rows solved 16 lanes each (MF_TINY_SOLVE=1,
    the default) against one warp each (MF_TINY_SOLVE=0): a forest of 2D
    9-point grids under AMF, whose lowest levels are all such fronts."""
    import scipy.sparse as sp
    mats = [tm.config3_matrix(int(s), seed=300 + i) for i, s in enumerate([8, 13, 21, 30, 17, 9, 25, 11])]
    A = sp.block_diag(mats).tocsc()
    P, S = mf.symbolic(A)
    B = tm.rhs(S.n, nrhs, seed=10 + nrhs)
    make = (lambda: mf.ldlt_(mf.ChordalLDLt(A, P, S))) if ldlt else (lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S)))
    X = both(monkeypatch, make, B, var="MF_TINY_SOLVE")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-13
    info, Xo, _ = oracle.factor_and_solve(A, P, S, B, int(ldlt))
    assert np.abs(X["1"] - Xo).max() <= 1e-9 * np.abs(Xo).max()


def test_tiny_fronts_mixed_refined(monkeypatch):
    A = tm.grid_laplacian(70, 65, stencil=9, seed=69)
    P, S = mf.symbolic(A)
    B = tm.rhs(S.n, 3, seed=11)
    X = both(monkeypatch, lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=True)), B, var="MF_TINY_SOLVE")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= 1e-12


@pytest.mark.parametrize("mixed", [False, True])
def test_step_kernels_with_programmatic_launch_equal_plain_launches(monkeypatch, mixed):
    """The per-step kernels launched for programmatic dependence (they issue
    their panel / inverse loads, then wait for the previous grid;
    MF_STEP_PDL=1, the default) against plain stream-ordered launches
    (MF_STEP_PDL=0), with the chain kernel off so every level runs the steps."""
    monkeypatch.setenv("MF_SOLVE_CHAIN", "0")
    A, P, S = grid(32, 30, 31, seed=71)
    B = tm.rhs(S.n, 4, seed=14)
    X = both(monkeypatch, lambda: mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=mixed)), B, var="MF_STEP_PDL")
    assert np.array_equal(X["0"], X["1"])
    assert tm.backward_error(A, X["1"], B).max() <= (1e-12 if mixed else 1e-13)
