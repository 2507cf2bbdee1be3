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

# elimination orders (0-based) under which the symbolic restatement yields
# the reference's displayed factor / tree; the displays fix the final order
CHOL_ORDER = np.array([3, 1, 4, 2, 5]) - 1
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


def test_cholesky_known_factor_and_solve():
    ka = KA["cholesky"]
    A = np.array(ka["A"])
    P, S = mf.symbolic(A, alg=CHOL_ORDER)
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
    P, S = mf.symbolic(A, alg=CHOL_ORDER)
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
    P, S = mf.symbolic(A, alg=CHOL_ORDER)
    Dval, Lval, _, _ = oracle.assemble(S, P.invp, A)
    info, *_ = oracle.chol_impl(S, Dval, Lval, 0)
    assert info > 0
    # factorize! maps the permuted column through perm (cholesky.jl:250-254)
    assert P.perm[info - 1] + 1 == 4
