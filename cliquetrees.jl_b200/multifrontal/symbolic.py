"""Symbolic factorization: ``ChordalSymbolic`` and ``Permutation``.

Mirrors src/Multifrontal.jl/src/chordal_symbolic.jl (struct :15-28,
``symbolic`` :68-91) and src/Multifrontal.jl/src/permutation.jl (:12-29).
The integer work runs in the C++ library ``libctsym.so``.  Arrays are kept
0-based; the ``*_1based`` helpers give the reference's 1-based view.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _native
from .sparse import SymmetricPattern, as_pattern


@dataclass
class Permutation:
    """A permutation matrix P with ``perm`` and ``invp`` (0-based).

    ``(P @ B)[invp[i]] = B[i]`` as in ``mul!(C, P, B)``
    (src/Multifrontal.jl/src/multiply.jl:277-280)."""
    perm: np.ndarray
    invp: np.ndarray

    @classmethod
    def from_perm(cls, perm):
        perm = np.ascontiguousarray(perm, dtype=np.int64)
        invp = np.empty_like(perm)
        invp[perm] = np.arange(perm.size, dtype=np.int64)
        return cls(perm, invp)


@dataclass
class ChordalSymbolic:
    """Symbolic factorization (chordal_symbolic.jl:15-28), 0-based.

    res(j) = columns resptr[j]:resptr[j+1]; sep(j) = septgt[sepptr[j]:sepptr[j+1]];
    rel has the pointers of sep and targets reltgt (position of each sep(j) row
    in bag(parent(j)) = res(p) ++ sep(p)); chd is the children CSR with the
    roots in list nfr; Dptr/Lptr are offsets of the diagonal (nn x nn) and
    off-diagonal (na x nn) blocks in Dval/Lval (column major)."""
    n: int
    nfr: int
    resptr: np.ndarray
    sepptr: np.ndarray
    septgt: np.ndarray
    reltgt: np.ndarray
    pnt: np.ndarray
    chdptr: np.ndarray
    chdtgt: np.ndarray
    idx: np.ndarray
    Dptr: np.ndarray
    Lptr: np.ndarray
    nMptr: int
    nMval: int
    nNval: int
    nFval: int

    @property
    def ndz(self) -> int:
        return int(self.Dptr[-1])

    @property
    def nlz(self) -> int:
        return int(self.Lptr[-1])

    def nn(self, j=None):
        d = np.diff(self.resptr)
        return d if j is None else int(d[j])

    def na(self, j=None):
        d = np.diff(self.sepptr)
        return d if j is None else int(d[j])

    def res(self, j):
        return np.arange(self.resptr[j], self.resptr[j + 1], dtype=np.int64)

    def sep(self, j):
        return self.septgt[self.sepptr[j]:self.sepptr[j + 1]]

    def rel(self, j):
        return self.reltgt[self.sepptr[j]:self.sepptr[j + 1]]

    def children(self, j):
        return self.chdtgt[self.chdptr[j]:self.chdptr[j + 1]]

    def roots(self):
        return self.children(self.nfr)

    def nnz(self) -> int:
        """Stored entries of the lower factor (chordal_symbolic.jl show)."""
        nn = self.nn()
        na = self.na()
        return int(np.sum(nn * (nn + 1) // 2 + nn * na))

    def factor_flops(self) -> float:
        """Algorithmic flops of one numeric factorization counted from the
        symbolic: sum over fronts of nn^3/3 + nn^2*na + nn*na^2."""
        nn = self.nn().astype(np.float64)
        na = self.na().astype(np.float64)
        return float(np.sum(nn ** 3 / 3.0 + nn * nn * na + nn * na * na))

    def levels(self):
        """Height of each front above the leaves (leaves = 0); fronts of one
        level have no ancestor relation and are factored together."""
        lvl = np.zeros(self.nfr, dtype=np.int64)
        for j in range(self.nfr):  # postorder: children before parents
            p = self.pnt[j]
            if p >= 0 and lvl[p] < lvl[j] + 1:
                lvl[p] = lvl[j] + 1
        return lvl


def _sym_from_handle(h) -> tuple[np.ndarray, np.ndarray, ChordalSymbolic]:
    lib = _native.symlib()
    sizes = np.zeros(9, dtype=np.int64)
    lib.ct_symbolic_sizes(h, _native.ptr64(sizes))
    n, nfr, nsep = int(sizes[0]), int(sizes[1]), int(sizes[2])
    order = np.empty(n, np.int64); invp = np.empty(n, np.int64)
    resptr = np.empty(nfr + 1, np.int64); sepptr = np.empty(nfr + 1, np.int64)
    septgt = np.empty(nsep, np.int64); reltgt = np.empty(nsep, np.int64)
    pnt = np.empty(nfr, np.int64); chdptr = np.empty(nfr + 2, np.int64)
    chdtgt = np.empty(nfr, np.int64); idx = np.empty(n, np.int64)
    Dptr = np.empty(nfr + 1, np.int64); Lptr = np.empty(nfr + 1, np.int64)
    p = _native.ptr64
    rc = lib.ct_symbolic_arrays(h, p(order), p(invp), p(resptr), p(sepptr), p(septgt), p(reltgt),
                                p(pnt), p(chdptr), p(chdtgt), p(idx), p(Dptr), p(Lptr))
    if rc != 0:
        raise RuntimeError("ct_symbolic_arrays failed")
    S = ChordalSymbolic(n, nfr, resptr, sepptr, septgt, reltgt, pnt, chdptr, chdtgt, idx,
                        Dptr, Lptr, int(sizes[5]), int(sizes[6]), int(sizes[7]), int(sizes[8]))
    return order, invp, S


def grid_nd_order(nx: int, ny: int, nz: int = 1, leaf: int = 8) -> np.ndarray:
    """Nested-dissection order of a grid by coordinate bisection (stands in
    for the METIS order; passed to ``symbolic`` as an explicit permutation)."""
    lib = _native.symlib()
    order = np.empty(nx * ny * nz, np.int64)
    rc = lib.ct_grid_nd_order(nx, ny, nz, leaf, _native.ptr64(order))
    if rc != 0:
        raise RuntimeError(lib.ct_last_error().decode())
    return order


def mindeg_order(pattern) -> np.ndarray:
    """Minimum-degree order (quotient graph, approximate external degrees;
    Amestoy, Davis & Duff 1996), computed by ``libctsym``."""
    pattern = as_pattern(pattern)
    lib = _native.symlib()
    order = np.empty(pattern.n, np.int64)
    rc = lib.ct_mindeg_order(pattern.n, _native.ptr64(pattern.colptr), _native.ptr64(pattern.rowval),
                             _native.ptr64(order))
    if rc != 0:
        raise RuntimeError(lib.ct_last_error().decode())
    return order


def amf_order(pattern) -> np.ndarray:
    """Approximate-minimum-fill order: the reference's default ``AMF()``
    (``AMFLib.amf`` on the simple graph of A, src/elimination_algorithms.jl:1556-1559,
    src/AMFLib.jl/src/AMFLib.jl:56-155 and hamf_impl! :703-1525), computed by
    ``libctsym``.  The adjacency lists are the columns of the symmetric
    pattern with rows ascending, as the reference reads a SparseMatrixCSC."""
    pattern = as_pattern(pattern)
    lib = _native.symlib()
    order = np.empty(pattern.n, np.int64)
    rc = lib.ct_amf_order(pattern.n, _native.ptr64(pattern.colptr), _native.ptr64(pattern.rowval),
                          _native.ptr64(order))
    if rc != 0:
        raise RuntimeError(lib.ct_last_error().decode())
    return order


def symbolic(A, alg="amf"):
    """``symbolic(A; alg)`` (chordal_symbolic.jl:68-91) -> (Permutation, ChordalSymbolic).

    ``alg`` is "amf" (the reference default ``AMF()``, elimination_algorithms.jl:2380),
    "mindeg" (minimum degree, an extra option), "natural", or an explicit
    order vector (0-based; order[i] = vertex eliminated i-th), as
    `permutation(weights, graph, order)` accepts (elimination_algorithms.jl:776-779)."""
    pat = as_pattern(A)
    n = pat.n
    if isinstance(alg, str):
        if alg == "amf":
            order = amf_order(pat)
        elif alg == "mindeg":
            order = mindeg_order(pat)
        elif alg == "natural":
            order = np.arange(n, dtype=np.int64)
        else:
            raise ValueError(f"unknown ordering {alg!r}")
    else:
        order = np.ascontiguousarray(alg, dtype=np.int64)
        if order.shape != (n,):
            raise ValueError("order has the wrong length")
    lib = _native.symlib()
    h = ctypes.c_void_p()
    rc = lib.ct_symbolic_create(n, _native.ptr64(pat.colptr), _native.ptr64(pat.rowval),
                                _native.ptr64(order), ctypes.byref(h))
    if rc != 0:
        raise ValueError(lib.ct_last_error().decode())
    try:
        perm, invp, S = _sym_from_handle(h)
    finally:
        lib.ct_symbolic_destroy(h)
    return Permutation(perm, invp), S
