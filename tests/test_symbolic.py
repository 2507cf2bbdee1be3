"""Invariants of the host symbolic restatement (ChordalSymbolic,
chordal_symbolic.jl:15-28, 302-378) on random graphs, checked against a
dense symbolic elimination."""
import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import testmatrices as tm


def random_graph(n, p, seed):
    rng = np.random.default_rng(seed)
    M = rng.random((n, n)) < p
    M = np.triu(M, 1)
    M = M | M.T
    return sp.csc_matrix(M.astype(float) + sp.eye(n))


def dense_structure(pattern, order):
    """Column structures of the Cholesky factor of P A P^T (boolean)."""
    n = pattern.shape[0]
    B = (abs(pattern).toarray() != 0)[np.ix_(order, order)]
    for k in range(n):
        nb = np.nonzero(B[k + 1:, k])[0] + k + 1
        B[np.ix_(nb, nb)] = True
    return np.tril(B)


@pytest.mark.parametrize("seed", range(6))
def test_structure_matches_dense_elimination(seed):
    n = 40
    A = random_graph(n, 0.08, seed)
    order = np.random.default_rng(100 + seed).permutation(n)
    P, S = mf.symbolic(A, alg=order)
    assert sorted(P.perm) == list(range(n))
    L = dense_structure(A, P.perm)
    # residuals contiguous, every column covered once
    assert S.resptr[0] == 0 and S.resptr[-1] == n and np.all(np.diff(S.resptr) > 0)
    for j in range(S.nfr):
        r = S.res(j)
        s = S.sep(j)
        assert np.all(np.diff(s) > 0) and (len(s) == 0 or s[0] > r[-1])
        # the bag of the first column is its structure; later columns drop one each
        for k, c in enumerate(r):
            want = np.nonzero(L[:, c])[0]
            got = np.concatenate([r[k:], s])
            np.testing.assert_array_equal(want, got)
        # maximal supernodes: the parent does not continue this front
        p = S.pnt[j]
        if p >= 0:
            assert p > j
            bagp = np.concatenate([S.res(p), S.sep(p)])
            np.testing.assert_array_equal(bagp[S.rel(j)], s)
    # Dptr / Lptr
    nn, na = S.nn(), S.na()
    np.testing.assert_array_equal(np.diff(S.Dptr), nn * nn)
    np.testing.assert_array_equal(np.diff(S.Lptr), nn * na)


def test_stack_bounds_match_lifo_simulation():
    A = tm.grid_laplacian(12, 9)
    P, S = mf.symbolic(A, alg=mf.grid_nd_order(12, 9, 1))
    ns, peak_n, peak_v, peak_nv = 1, 1, 0, 0
    mv = nv = 0
    for j in range(S.nfr):
        for c in S.children(j):
            ma = S.na(c)
            ns -= 1; mv -= ma * ma; nv -= ma
        na = S.na(j)
        if na > 0:
            ns += 1; mv += na * na; nv += na
            peak_n, peak_v, peak_nv = max(peak_n, ns), max(peak_v, mv), max(peak_nv, nv)
    assert (S.nMptr, S.nMval, S.nNval) == (peak_n, peak_v, peak_nv)
    assert S.nFval == int((S.nn() + S.na()).max())


def test_children_ascending_and_roots_last_list():
    A = random_graph(60, 0.03, 7)  # likely disconnected: several roots
    P, S = mf.symbolic(A, alg="natural")
    for j in range(S.nfr + 1):
        ch = S.children(j)
        assert np.all(np.diff(ch) > 0)
    roots = S.roots()
    assert np.all(S.pnt[roots] == -1)
    assert len(roots) == int(np.sum(S.pnt == -1))


def test_invalid_order_rejected():
    A = tm.grid_laplacian(4, 4)
    with pytest.raises(ValueError):
        mf.symbolic(A, alg=np.zeros(16, dtype=np.int64))


def test_grid_nd_order_is_permutation():
    for dims in [(5, 7, 1), (6, 5, 4), (1, 1, 1), (16, 16, 16)]:
        o = mf.grid_nd_order(*dims)
        assert sorted(o) == list(range(int(np.prod(dims))))


def test_mindeg_order_is_a_good_permutation():
    """Minimum-degree order (stand-in for the reference's AMF): a valid
    permutation, deterministic, and far less fill than the natural order on
    2D/3D grids and on a quasidefinite KKT matrix."""
    from multifrontal import testmatrices as tm
    for A in (tm.config1(), tm.grid_laplacian(12, 11, 10), tm.config4(side=8, m=150, seed=3)):
        n = A.shape[0]
        o = mf.mindeg_order(A)
        assert np.array_equal(np.sort(o), np.arange(n))
        assert np.array_equal(o, mf.mindeg_order(A))
        _, S = mf.symbolic(A, alg=o)
        _, Sn = mf.symbolic(A, alg="natural")
        assert S.nnz() < 0.7 * Sn.nnz()


def test_mindeg_on_a_path_and_a_star():
    """Known answers: a path is eliminated without fill; a star keeps its
    centre until only one leaf is left (every leaf has degree 1, the centre
    degree n - 1 - eliminated leaves)."""
    import scipy.sparse as sp
    n = 9
    path = sp.diags([np.ones(n - 1), np.ones(n - 1)], [-1, 1], shape=(n, n), format="csc")
    _, S = mf.symbolic(path + sp.eye(n, format="csc"), alg="mindeg")
    assert S.nnz() == 2 * n - 1
    rows = np.arange(1, n)
    star = sp.csc_matrix((np.ones(n - 1), (rows, np.zeros(n - 1, int))), shape=(n, n))
    star = star + star.T + sp.eye(n, format="csc")
    o = mf.mindeg_order(star)
    assert 0 in o[-2:]
    _, S = mf.symbolic(star, alg=o)
    assert S.nnz() == 2 * n - 1
