"""Sparse-matrix plumbing on the host: symmetric patterns, the symmetric
permutation of the lower triangle and the flat index map from A's stored
entries into the factor storage.

Reference:
  sympermute(A, invp, src, tgt)        src/Multifrontal.jl/src/utils.jl:147-219
  copyto!(::ChordalTriangular, ::SparseMatrixCSC)
                                       src/Multifrontal.jl/src/chordal_triangular.jl:852-893
  flatindices(S, B, Val(:L))           src/Multifrontal.jl/src/chordal_symbolic.jl:595-660
  flatindices(invp, S, A, uplo)        src/Multifrontal.jl/src/chordal_symbolic.jl:731-752
All indices 0-based.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp


@dataclass
class SymmetricPattern:
    n: int
    colptr: np.ndarray
    rowval: np.ndarray


def to_csc(A) -> sp.csc_matrix:
    if sp.issparse(A):
        C = sp.csc_matrix(A)
    else:
        C = sp.csc_matrix(np.asarray(A, dtype=np.float64))
    if C.shape[0] != C.shape[1]:
        raise ValueError("matrix must be square")
    C.sum_duplicates()
    C.sort_indices()
    return C


def as_pattern(A) -> SymmetricPattern:
    """Symmetric pattern of A (union of both triangles), CSC int64."""
    if isinstance(A, SymmetricPattern):
        return A
    C = to_csc(A)
    n = C.shape[0]
    P = (abs(C) + abs(C).T).tocsc()
    P.sort_indices()
    return SymmetricPattern(n, P.indptr.astype(np.int64), P.indices.astype(np.int64))


def lower_triangle(A) -> sp.csc_matrix:
    """The lower triangle of a symmetric matrix given by either triangle or
    both (the check=false / Hermitian(A, :L) paths of chordal_factorization.jl:205-219)."""
    C = to_csc(A)
    strict_up = sp.triu(C, k=1, format="csc")
    strict_lo = sp.tril(C, k=-1, format="csc")
    if strict_up.nnz == 0 or (C - C.T).count_nonzero() == 0:
        lo = sp.tril(C, format="csc")
    elif strict_lo.nnz == 0:
        lo = sp.csc_matrix(sp.triu(C, format="csc").T)
    else:
        raise ValueError("matrix is neither symmetric nor triangular")
    lo.sort_indices()
    return lo


def sympermute_lower(L: sp.csc_matrix, invp: np.ndarray):
    """Lower triangle of P A P^T from the lower triangle of A, rows sorted,
    plus, for every stored entry of the result, the index of the entry of L
    it came from (utils.jl:147-219 with src = tgt = 'L')."""
    L = sp.csc_matrix(L)
    n = L.shape[0]
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(L.indptr))
    rows = L.indices.astype(np.int64)
    pi, pj = invp[rows], invp[cols]
    hi = np.maximum(pi, pj)
    lo = np.minimum(pi, pj)
    # column = lo (smaller new label), row = hi
    key = lo * n + hi
    order = np.argsort(key, kind="stable")
    colptr = np.zeros(n + 1, np.int64)
    np.add.at(colptr, lo + 1, 1)
    colptr = np.cumsum(colptr)
    return colptr, hi[order], order


def flatindices_lower(S, colptr: np.ndarray, rowval: np.ndarray) -> np.ndarray:
    """For each stored entry (row, col) of the permuted lower triangle, its
    0-based flat slot in [Dval; Lval] (flatindices(S, B, Val(:L)),
    chordal_symbolic.jl:595-660).  Dval block of front j is nn x nn column
    major at Dptr[j]; Lval block is na x nn at ndz + Lptr[j]."""
    n = S.n
    nnz = rowval.size
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(colptr))
    front = S.idx[cols]
    r0 = S.resptr[front]
    r1 = S.resptr[front + 1]
    nn = r1 - r0
    na = S.sepptr[front + 1] - S.sepptr[front]
    c = cols - r0
    out = np.empty(nnz, np.int64)
    inD = rowval < r1
    out[inD] = S.Dptr[front[inD]] + (rowval[inD] - r0[inD]) + c[inD] * nn[inD]
    off = ~inD
    if np.any(off):
        # position of the row in sep(front)
        fr = front[off]
        rw = rowval[off]
        pos = np.empty(fr.size, np.int64)
        # searchsorted per front: septgt is sorted within each front's slice
        # search in the concatenated array with a front-specific offset key
        big = np.int64(n + 1)
        key_tgt = np.repeat(np.arange(S.nfr, dtype=np.int64), np.diff(S.sepptr)) * big + S.septgt
        key = fr * big + rw
        loc = np.searchsorted(key_tgt, key)
        ok = (loc < key_tgt.size)
        ok[ok] = key_tgt[loc[ok]] == key[ok]
        if not np.all(ok):
            raise ValueError("matrix entry outside the symbolic pattern")
        pos = loc - S.sepptr[fr]
        out[off] = S.ndz + S.Lptr[fr] + pos + c[off] * na[off]
    return out


def assembly_map(S, invp: np.ndarray, A):
    """(lower CSC of A, slot) where slot[k] is the flat [Dval; Lval] index
    of A's k-th stored lower-triangle entry (flatindices(invp, S, A, Val(:L)),
    chordal_symbolic.jl:731-752).  The values then assemble as
    flat[slot[k]] = L.data[k]."""
    L = lower_triangle(A)
    colptr, rowval, src = sympermute_lower(L, invp)
    slot_sorted = flatindices_lower(S, colptr, rowval)
    slot = np.empty_like(slot_sorted)
    slot[src] = slot_sorted
    return L, slot
