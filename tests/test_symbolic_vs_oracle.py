"""The product's host symbolic analysis (libctsym: AMF, supernodes, clique
tree, ChordalSymbolic) against the oracle's own restatement (oracle/sym_oracle.c),
integer-exact, on the reference's known answers and on seeded graphs of the
benchmark shapes.  Both restate the reference; they share no code."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

import multifrontal as mf
from multifrontal import testmatrices as tm
from oracle import oracle

KA = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "known_answers.json")))

FIELDS = ["resptr", "sepptr", "septgt", "reltgt", "pnt", "chdptr", "chdtgt", "idx", "Dptr", "Lptr"]


def random_graph(n, deg, seed):
    rng = np.random.default_rng(seed)
    m = n * deg // 2
    i = rng.integers(0, n, m)
    j = rng.integers(0, n, m)
    A = sp.coo_matrix((np.ones(m), (i, j)), shape=(n, n))
    A = (A + A.T + sp.eye(n)).tocsc()
    A.data[:] = 1.0
    return A


def cases():
    yield "amf8", np.array(KA["amf"]["graph"], float)
    yield "vda17", np.array(KA["maximal17"]["graph"], float)
    yield "grid2d", tm.grid_laplacian(37, 23, seed=1)
    yield "grid2d9", tm.config3_matrix(31, seed=2)
    yield "grid3d", tm.grid_laplacian(11, 9, 8, seed=3)
    yield "kkt", tm.config4(side=8, m=128, seed=4)
    for s in range(6):
        yield f"random{s}", random_graph(300 + 97 * s, 2 + s, seed=s)
    yield "disconnected", sp.block_diag([tm.grid_laplacian(5, 4), sp.eye(3), tm.grid_laplacian(3, 3, 3)],
                                        format="csc")


@pytest.mark.parametrize("name,A", list(cases()), ids=[c[0] for c in cases()])
def test_amf_order_matches_oracle(name, A):
    assert np.array_equal(mf.amf_order(A), oracle.amf_order(A))


@pytest.mark.parametrize("name,A", list(cases()), ids=[c[0] for c in cases()])
def test_symbolic_matches_oracle(name, A):
    for alg in ("amf", "natural"):
        P, S = mf.symbolic(A, alg=alg)
        Po, So = oracle.symbolic(A, alg="amf" if alg == "amf" else np.arange(A.shape[0]))
        assert np.array_equal(P.perm, Po.perm), alg
        assert S.nfr == So.nfr
        for f in FIELDS:
            assert np.array_equal(getattr(S, f), getattr(So, f)), (alg, f)
        for f in ("nMptr", "nMval", "nNval", "nFval"):
            assert getattr(S, f) == getattr(So, f), (alg, f)


def test_oracle_assembly_matches_product_slot_map():
    from multifrontal.sparse import assembly_map
    A = tm.config4(side=6, m=60, seed=8)
    P, S = mf.symbolic(A)
    _, slot = assembly_map(S, P.invp, A)
    _, _, _, slot_o = oracle.assemble(S, P.invp, A)
    assert np.array_equal(slot, slot_o)


def test_oracle_symbolic_large_grid_matches():
    """A config-2-shaped grid (smaller side) under AMF: the two restatements
    agree on every array."""
    A = tm.config2(side=24, seed=2)
    P, S = mf.symbolic(A)
    Po, So = oracle.symbolic(A)
    assert np.array_equal(P.perm, Po.perm)
    for f in FIELDS:
        assert np.array_equal(getattr(S, f), getattr(So, f)), f
