"""The oracle and the symbolic restatement against the reference's own
published examples (tests/golden/known_answers.json, extracted from the
reference READMEs by tests/golden/make_known_answers.py)."""
import json
import os

import numpy as np
import pytest

import multifrontal as mf
from oracle import oracle

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))

# elimination order (0-based) under which the symbolic restatement yields
# the README's clique tree for alg=MF() (MF is not restated; the display
# fixes the final order)
TREE_ORDER = np.array([1, 4, 2, 5, 8, 3, 6, 7]) - 1


def dense_factor(S, Dval, Lval):
    n = S.n
    L = np.zeros((n, n))
    for j in range(S.nfr):
        r = S.res(j); s = S.sep(j); nn = len(r); na = len(s)
        D = Dval[S.Dptr[j]:S.Dptr[j] + nn * nn].reshape(nn, nn, order="F")
        Lj = Lval[S.Lptr[j]:S.Lptr[j] + nn * na].reshape(na, nn, order="F")
        for c in range(nn):
            L[r[c:], r[c]] = D[c:, c]
            L[s, r[c]] = Lj[:, c]
    return L


def test_amf_known_order():
    """AMFLib README: amf(8, graph.colptr, graph.rowval) -> perm (src/AMFLib.jl/README.md)."""
    G = np.array(KA["amf"]["graph"], float)
    assert list(mf.amf_order(G) + 1) == KA["amf"]["perm"]


def test_default_ordering_is_amf():
    """symbolic(A) orders with AMF() by default (elimination_algorithms.jl:2380);
    supernode relabelling keeps this order for the 8-vertex graph."""
    G = np.array(KA["amf"]["graph"], float)
    P, S = mf.symbolic(G)
    assert list(P.perm + 1) == KA["amf"]["perm"]
    # every bag of the clique tree is a clique of the filled graph in
    # elimination order: residual columns contiguous, separators after them
    for j in range(S.nfr):
        assert np.all(S.sep(j) >= S.resptr[j + 1])


def test_maximal_clique_tree_of_the_17_vertex_graph():
    """test/core.jl "vandenberghe and andersen", snd = Maximal() (Figure 4.7
    left): parent indices, residuals and separators under the order 1:17."""
    K = KA["maximal17"]
    G = np.array(K["graph"], float)
    P, S = mf.symbolic(G, alg=np.array(K["order"]) - 1)
    assert S.nfr == len(K["parent"])
    assert [None if p < 0 else int(p) + 1 for p in S.pnt] == K["parent"]
    assert [list(map(int, P.perm[S.res(j)] + 1)) for j in range(S.nfr)] == K["residual_labels"]
    assert [list(map(int, P.perm[S.sep(j)] + 1)) for j in range(S.nfr)] == K["separator_labels"]


def test_cholesky_known_factor_and_solve():
    """README: cholesky!(ChordalCholesky(A)) with the default ordering (AMF)."""
    ka = KA["cholesky"]
    A = np.array(ka["A"])
    P, S = mf.symbolic(A)
    assert list(P.perm + 1) == [3, 1, 2, 4, 5]
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 0)
    assert info == 0
    want = np.nan_to_num(np.array(ka["L"]), nan=0.0)
    np.testing.assert_array_equal(dense_factor(S, Dval, Lval), want)
    info, x, _ = oracle.factor_and_solve(A, P, S, np.array(ka["b"]), 0)
    np.testing.assert_array_equal(x, np.array(ka["x"]))


@pytest.mark.parametrize("use_signs", [False, True])
def test_ldlt_known_factor_and_solve(use_signs):
    ka = KA["ldlt"]
    A = np.array(ka["A"])
    P, S = mf.symbolic(A)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    signs = np.array(ka["signs"])[P.perm] if use_signs else None
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 1, signs=signs)
    assert info == 0
    Lw = np.nan_to_num(np.array(ka["L_signs" if use_signs else "L"]), nan=0.0)
    L = dense_factor(S, Dval, Lval)
    np.fill_diagonal(L, 1.0)  # unit diagonal is implied (potrf.jl:10-13)
    np.testing.assert_array_equal(L, Lw)
    np.testing.assert_array_equal(d, np.array(ka["d_signs" if use_signs else "d"]))
    info, x, _ = oracle.factor_and_solve(A, P, S, np.array(ka["b"]), 1)
    np.testing.assert_array_equal(x, np.array(ka["x"]))


def test_cliquetree_known_tree():
    G = np.array(KA["amf"]["graph"], float)
    P, S = mf.symbolic(G, alg=TREE_ORDER)
    bags = [tuple(int(v) + 1 for v in list(S.res(j)) + list(S.sep(j))) for j in range(S.nfr)]
    got = {(bags[j], None if S.pnt[j] < 0 else bags[S.pnt[j]]) for j in range(S.nfr)}
    want = {(tuple(nd["bag"]), None if nd["parent"] is None else tuple(nd["parent"])) for nd in KA["cliquetree_mf"]}
    assert got == want
    # the display lists the nodes in preorder with ascending children; our
    # postorder must list children before parents and siblings ascending
    order = [bags[j] for j in range(S.nfr)]
    assert order == [(1, 5), (2, 3), (3, 5, 7), (4, 5, 8), (5, 7, 8), (6, 7, 8)]


def test_failure_info_is_first_bad_pivot_in_original_order():
    # make the 5x5 example indefinite at original vertex 4
    A = np.array(KA["cholesky"]["A"])
    A[3, 3] = -1.0
    P, S = mf.symbolic(A)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, *_ = oracle.chol_impl(S, Dval, Lval, 0)
    assert info > 0
    # factorize! maps the permuted column through perm (cholesky.jl:250-254)
    assert P.perm[info - 1] + 1 == 4


def test_selinv_known_answer():
    """selinv.jl docstring: selinv!(cholesky!(ChordalCholesky(A))) with the
    default ordering, displayed in elimination order."""
    ka = KA["selinv"]
    A = np.array(ka["A"])
    P, S = oracle.symbolic(A)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 0)
    assert info == 0
    Zd, Zl = oracle.selinv(S, Dval, Lval)
    want = np.nan_to_num(np.array(ka["Z"]), nan=0.0)
    np.testing.assert_allclose(dense_factor(S, Zd, Zl), want, rtol=0, atol=1e-15)


def test_selinv_oracle_equals_inverse_on_the_pattern():
    """The oracle's selected inverse equals A^-1 on the pattern of L."""
    from multifrontal import testmatrices as tm
    A = tm.grid_laplacian(9, 8, 3, seed=4)
    P, S = oracle.symbolic(A)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 0)
    Zd, Zl = oracle.selinv(S, Dval, Lval)
    Z = dense_factor(S, Zd, Zl)
    mask = dense_factor(S, np.ones_like(Dval), np.ones_like(Lval)) != 0
    Ai = np.linalg.inv(A.toarray())[np.ix_(P.perm, P.perm)]
    assert np.abs((Z - Ai)[mask]).max() <= 1e-12 * np.abs(Ai).max()


def test_dynamic_regularization_known_answer():
    """dynamic_regularization.jl docstring: cholesky!(ChordalCholesky(A);
    reg=DynamicRegularization()) of an indefinite matrix; Matrix(F) is
    printed to six significant digits."""
    ka = KA["dynamic_regularization"]
    A = np.array(ka["A"])
    P, S = oracle.symbolic(A)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, Dval, Lval, d = oracle.chol_impl(S, Dval, Lval, 0, reg=(-1.0, -1.0))
    assert info == 0
    L = dense_factor(S, Dval, Lval)
    B = (L @ L.T)[np.ix_(P.invp, P.invp)]
    np.testing.assert_allclose(B, np.array(ka["B"]), rtol=5e-6)
