"""Host side of batching: the ChordalSymbolic of a block-diagonal batch
is the concatenation of the per-matrix ones (no GPU needed)."""
import numpy as np

import multifrontal as mf
from multifrontal import batch
from multifrontal import testmatrices as tm
from oracle import oracle


def _batch(m, seed=0, lo=6, hi=18):
    rng = np.random.default_rng(seed)
    sides = rng.integers(lo, hi + 1, size=m)
    mats = [tm.config3_matrix(int(s), seed=100 + i) for i, s in enumerate(sides)]
    orders = [mf.grid_nd_order(int(s), int(s), 1) for s in sides]
    return mats, orders


def test_block_symbolic_is_consistent():
    mats, orders = _batch(5, seed=3)
    parts = [mf.symbolic(A, alg=o) for A, o in zip(mats, orders)]
    P, S, off = batch.block_symbolic(parts)
    assert S.n == sum(A.shape[0] for A in mats) and off[-1] == S.n
    assert S.nfr == sum(s.nfr for _, s in parts)
    assert S.roots().size == sum(s.roots().size for _, s in parts)
    assert np.all(np.diff(S.resptr) > 0)
    # every front's parent comes later (postorder kept)
    assert np.all((S.pnt < 0) | (S.pnt > np.arange(S.nfr)))



def test_block_symbolic_equals_symbolic_of_block_matrix():
    """The concatenated symbolic has the fronts the symbolic analysis finds
    for the block-diagonal matrix with the concatenated order (the analysis
    may visit the trees of the forest in another order)."""
    import scipy.sparse as sp
    mats, orders = _batch(4, seed=5)
    parts = [mf.symbolic(A, alg=o) for A, o in zip(mats, orders)]
    P, S, off = batch.block_symbolic(parts)
    order = np.concatenate([o + off[i] for i, o in enumerate(orders)])
    P2, S2 = mf.symbolic(sp.block_diag(mats, format="csc"), alg=order)
    assert S.nfr == S2.nfr and S.nnz() == S2.nnz()
    assert sorted(zip(S.nn(), S.na())) == sorted(zip(S2.nn(), S2.na()))
    assert abs(S.factor_flops() - S2.factor_flops()) <= 1e-9 * S2.factor_flops()
    # the same partition of columns into fronts, in original labels
    fronts = sorted(tuple(sorted(P.perm[S.resptr[j]:S.resptr[j + 1]])) for j in range(S.nfr))
    fronts2 = sorted(tuple(sorted(P2.perm[S2.resptr[j]:S2.resptr[j + 1]])) for j in range(S2.nfr))
    assert fronts == fronts2


def test_batch_oracle_matches_per_matrix_oracle():
    """The CPU oracle on the concatenated symbolic reproduces each matrix's
    own factorization bit for bit (the forest is factored tree by tree)."""
    import scipy.sparse as sp
    mats, orders = _batch(3, seed=6)
    parts = [mf.symbolic(A, alg=o) for A, o in zip(mats, orders)]
    P, S, off = batch.block_symbolic(parts)
    Ab = sp.block_diag(mats, format="csc")
    Bb = tm.rhs(S.n, 2, seed=9)
    info, Xb, _ = oracle.factor_and_solve(Ab, P, S, Bb, 0)
    assert info == 0
    for i, (A, (Pi, Si)) in enumerate(zip(mats, parts)):
        info, Xi, _ = oracle.factor_and_solve(A, Pi, Si, Bb[off[i]:off[i + 1]], 0)
        assert np.array_equal(Xi, Xb[off[i]:off[i + 1]])
