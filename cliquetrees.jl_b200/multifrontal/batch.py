"""Many independent matrices factored and solved together as one forest.

The reference factors one matrix per ``ChordalFactorization``.  For a batch
of independent matrices A_1 .. A_m, the block-diagonal matrix
diag(A_1, ..., A_m) has the forest of the individual elimination trees as
its elimination tree, so concatenating the per-matrix ``ChordalSymbolic``
arrays -- columns and fronts offset, children lists kept, every tree's root
in the root list -- gives a valid ``ChordalSymbolic`` of the block matrix
(chordal_symbolic.jl:15-28; the LIFO bounds nMptr/nMval/nNval/nFval of a
forest processed tree after tree are the maxima over the trees).

The device plan then schedules tree level by tree level across all
matrices: every grouped launch (small fronts, extend-add, blocked steps,
solves) covers the fronts of one level of every matrix, and the factor and
the solve of the whole batch are one CUDA graph each.  Each matrix is a
segment of rows; the mixed form's refinement measures the normwise backward
error of every matrix separately and runs until the worst one meets the
tolerance.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

from . import _native
from ._native import check, ptr64
from .factorization import ChordalCholesky, ChordalLDLt, ldiv
from .symbolic import ChordalSymbolic, Permutation, symbolic


def block_symbolic(parts):
    """Concatenate [(Permutation, ChordalSymbolic), ...] into the
    (Permutation, ChordalSymbolic) of the block-diagonal matrix, plus the
    column offset of every block (length m + 1)."""
    if not parts:
        raise ValueError("empty batch")
    ns = np.array([S.n for _, S in parts], dtype=np.int64)
    nfs = np.array([S.nfr for _, S in parts], dtype=np.int64)
    coff = np.concatenate([[0], np.cumsum(ns)])
    foff = np.concatenate([[0], np.cumsum(nfs)])
    n, nfr = int(coff[-1]), int(foff[-1])
    perm = np.concatenate([P.perm + coff[i] for i, (P, _) in enumerate(parts)])
    resptr = np.concatenate([[0]] + [S.resptr[1:] + coff[i] for i, (_, S) in enumerate(parts)])
    nsep = np.array([S.sepptr[-1] for _, S in parts], dtype=np.int64)
    soff = np.concatenate([[0], np.cumsum(nsep)])
    sepptr = np.concatenate([[0]] + [S.sepptr[1:] + soff[i] for i, (_, S) in enumerate(parts)])
    septgt = np.concatenate([S.septgt + coff[i] for i, (_, S) in enumerate(parts)])
    reltgt = np.concatenate([S.reltgt for _, S in parts])
    pnt = np.concatenate([np.where(S.pnt >= 0, S.pnt + foff[i], -1) for i, (_, S) in enumerate(parts)])
    idx = np.concatenate([S.idx + foff[i] for i, (_, S) in enumerate(parts)])
    ndz = np.array([S.Dptr[-1] for _, S in parts], dtype=np.int64)
    nlz = np.array([S.Lptr[-1] for _, S in parts], dtype=np.int64)
    doff = np.concatenate([[0], np.cumsum(ndz)])
    loff = np.concatenate([[0], np.cumsum(nlz)])
    Dptr = np.concatenate([[0]] + [S.Dptr[1:] + doff[i] for i, (_, S) in enumerate(parts)])
    Lptr = np.concatenate([[0]] + [S.Lptr[1:] + loff[i] for i, (_, S) in enumerate(parts)])
    # children lists of the fronts, then all roots
    kids, roots = [], []
    counts = np.empty(nfr + 1, np.int64)
    for i, (_, S) in enumerate(parts):
        c = np.diff(S.chdptr)
        counts[foff[i]:foff[i + 1]] = c[:S.nfr]
        kids.append(S.chdtgt[:S.chdptr[S.nfr]] + foff[i])
        roots.append(S.chdtgt[S.chdptr[S.nfr]:S.chdptr[S.nfr + 1]] + foff[i])
    roots = np.concatenate(roots)
    counts[nfr] = roots.size
    chdptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    chdtgt = np.concatenate(kids + [roots]).astype(np.int64)
    S = ChordalSymbolic(n, nfr, resptr.astype(np.int64), sepptr.astype(np.int64), septgt.astype(np.int64),
                        reltgt.astype(np.int64), pnt.astype(np.int64), chdptr, chdtgt, idx.astype(np.int64),
                        Dptr.astype(np.int64), Lptr.astype(np.int64),
                        max(S.nMptr for _, S in parts), max(S.nMval for _, S in parts),
                        max(S.nNval for _, S in parts), max(S.nFval for _, S in parts))
    return Permutation.from_perm(perm), S, coff


class BatchedFactorization:
    """A batch of independent symmetric matrices factored as one forest.

    ``mats``: list of sparse matrices; ``orders``: per-matrix ordering
    (anything ``symbolic(A, alg=...)`` accepts) or one value for all.
    ``ldlt=True`` gives ChordalLDLt semantics, else ChordalCholesky.
    ``mixed=True``: FP32 fronts + FP64 refinement to per-matrix backward
    error ``tol``."""

    def __init__(self, mats, orders="amf", *, ldlt=False, mixed=False, tol=1e-12, maxit=100, device=0,
                 nrhs_cap=16, symbolics=None):
        self.m = len(mats)
        if symbolics is None:
            if not isinstance(orders, (list, tuple)):
                orders = [orders] * self.m
            symbolics = [symbolic(A, alg=o) for A, o in zip(mats, orders)]
        self.parts = symbolics
        self.P, self.S, self.offsets = block_symbolic(symbolics)
        self.A = sp.block_diag([sp.csc_matrix(A) for A in mats], format="csc")
        cls = ChordalLDLt if ldlt else ChordalCholesky
        self.F = cls(self.A, self.P, self.S, device=device, nrhs_cap=nrhs_cap, mixed=mixed, tol=tol, maxit=maxit)
        lib = _native.gpulib()
        check(lib.mf_set_segments(self.F._handle.h, self.m, ptr64(np.ascontiguousarray(self.offsets))),
              "mf_set_segments")

    @property
    def n(self):
        return self.S.n

    def refresh(self, mats):
        """New values on the same patterns (the value-refresh path)."""
        self.A = sp.block_diag([sp.csc_matrix(A) for A in mats], format="csc")
        self.F.copyto(self.A)
        return self

    def factorize(self, *, check=True, signs=None):
        from .factorization import cholesky_, ldlt_
        if isinstance(self.F, ChordalLDLt):
            ldlt_(self.F, signs=signs, check=check)
        else:
            cholesky_(self.F, check=check)
        return self

    def autotune(self, reps=3):
        """Mixed form: per-level tcgen05/FFMA choice timed on the current values
        (``ChordalFactorization.autotune``); factorize again afterwards."""
        return self.F.autotune(reps)

    @property
    def info(self):
        return self.F.info

    def failed_matrix(self):
        """Index of the matrix holding the first rejected pivot, or -1."""
        if self.F.info == 0:
            return -1
        col = self.F.info - 1
        return int(np.searchsorted(self.offsets, col, side="right") - 1)

    def solve(self, Bs):
        """Solve every matrix against its right-hand sides; ``Bs`` is a list of
        (n_i x k) arrays with the same k, or one (sum n_i x k) array."""
        if isinstance(Bs, (list, tuple)):
            B = np.concatenate([np.asarray(b, dtype=np.float64).reshape(b.shape[0], -1) for b in Bs], axis=0)
            X = ldiv(self.F, B)
            return [X[self.offsets[i]:self.offsets[i + 1]] for i in range(self.m)]
        return ldiv(self.F, Bs)

    def segment_errors(self):
        """Per-matrix backward error of the last refined solve (worst column), mixed form only."""
        out = np.zeros(self.m, np.float64)
        check(_native.gpulib().mf_segment_errors(self.F._handle.h, _native.ptrd(out)), "mf_segment_errors")
        return out

    def close(self):
        self.F.close()
