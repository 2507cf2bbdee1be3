"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for the multifrontal numeric phase.

Python driver around ``mf_oracle.c`` (a C restatement of CliqueTrees.jl's
chol_impl!/div_impl!, see the header of that file for the line-by-line
citations) and ``sym_oracle.c`` (the reference's symbolic analysis: AMF and
the chain to a ChordalSymbolic).  Only tests, ``__graft_entry__.smoke()``
and the CPU legs of ``bench.py`` may import this module; the product never
does, and this module imports nothing from the product.

Parity status: the reference is Julia and cannot run in this environment,
so the restatement is pinned by the in-repository known answers (the 5x5
Cholesky/LDLt factors and solves of the reference's docstrings and
READMEs) and by backward-error checks; bitwise parity with a Julia run is
unpinned.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libmforacle.so")
SRC = os.path.join(HERE, "mf_oracle.c")
SYM_SRC = os.path.join(HERE, "sym_oracle.c")

_i64 = ctypes.c_int64
_p64 = ctypes.POINTER(ctypes.c_int64)
_pd = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    stale = not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(SRC), os.path.getmtime(SYM_SRC))
    if force or stale:
        # -ffp-contract=off: the AMF fill score rounds as separate multiply and subtract
        subprocess.run(["gcc", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB, SRC,
                        SYM_SRC, "-ldl", "-lm"], check=True)
    return LIB


def openblas_path() -> str:
    import scipy
    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas*.so"))
    if not libs:
        raise RuntimeError("scipy-bundled OpenBLAS not found")
    return os.path.abspath(libs[0])


_lib = None


def lib(nthreads: int = 1):
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        L.mfo_init.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.mfo_init.restype = ctypes.c_int
        L.mfo_chol_impl.argtypes = [_i64, _i64] + [_p64] * 7 + [_i64, _i64, _i64, ctypes.c_int, _pd, _pd, _pd, _pd]
        L.mfo_chol_impl.restype = ctypes.c_int64
        L.mfo_div_impl.argtypes = [_i64, _i64] + [_p64] * 7 + [_i64, _i64, _i64, ctypes.c_int, _pd, _pd, _pd, _pd,
                                                               _i64, _i64, ctypes.c_int]
        L.mfo_div_impl.restype = ctypes.c_int
        L.mfo_set_regularization.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.mfo_set_regularization.restype = None
        L.mfo_selinv.argtypes = [_i64, _i64] + [_p64] * 7 + [_i64, _i64, _i64, _pd, _pd]
        L.mfo_selinv.restype = ctypes.c_int
        L.mfo_amf_order.argtypes = [_i64, _p64, _p64, _p64]
        L.mfo_amf_order.restype = ctypes.c_int
        L.mfo_symbolic_create.argtypes = [_i64, _p64, _p64, _p64]
        L.mfo_symbolic_create.restype = ctypes.c_void_p
        L.mfo_symbolic_free.argtypes = [ctypes.c_void_p]
        L.mfo_symbolic_sizes.argtypes = [ctypes.c_void_p, _p64]
        L.mfo_symbolic_arrays.argtypes = [ctypes.c_void_p] + [_p64] * 11
        rc = L.mfo_init(openblas_path().encode(), nthreads)
        if rc != 0:
            raise RuntimeError(f"mfo_init failed ({rc})")
        _lib = L
    else:
        _lib.mfo_init(openblas_path().encode(), nthreads)
    return _lib


def set_threads(n: int):
    lib(n)


def _p(a):
    return None if a is None else a.ctypes.data_as(_p64)


def _d(a):
    return None if a is None else a.ctypes.data_as(_pd)


def chol_impl(S, Dval, Lval, diag: int, signs=None, d=None, reg=None):
    """Run the oracle factorization in place.  Returns (info, d).  ``reg``:
    None (NoRegularization) or (delta, epsilon) for DynamicRegularization
    (negative values take the defaults)."""
    L = lib()
    if reg is None:
        L.mfo_set_regularization(0, -1.0, -1.0)
    else:
        L.mfo_set_regularization(1, float(reg[0]), float(reg[1]))
    Dval = np.ascontiguousarray(Dval, dtype=np.float64)
    Lval = np.ascontiguousarray(Lval, dtype=np.float64)
    if d is None:
        d = np.zeros(max(S.n, 1), np.float64)
    sg = None if signs is None else np.ascontiguousarray(signs, dtype=np.float64)
    info = L.mfo_chol_impl(S.n, S.nfr, _p(S.resptr), _p(S.sepptr), _p(S.reltgt), _p(S.chdptr), _p(S.chdtgt),
                           _p(S.Dptr), _p(S.Lptr), S.nMptr, S.nMval, S.nFval, diag, _d(Dval), _d(Lval), _d(d),
                           _d(sg))
    L.mfo_set_regularization(0, -1.0, -1.0)
    if info < 0:
        raise MemoryError("oracle allocation failed")
    return int(info), Dval, Lval, d


def selinv(S, Dval, Lval):
    """selinv! (selinv.jl:38-424) of a Cholesky factor in place: returns
    (Dval, Lval) holding A^{-1} on the pattern of L."""
    L = lib()
    Dval = np.ascontiguousarray(Dval, dtype=np.float64).copy()
    Lval = np.ascontiguousarray(Lval, dtype=np.float64).copy()
    rc = L.mfo_selinv(S.n, S.nfr, _p(S.resptr), _p(S.sepptr), _p(S.reltgt), _p(S.chdptr), _p(S.chdtgt),
                      _p(S.Dptr), _p(S.Lptr), S.nMptr, S.nMval, S.nFval, _d(Dval), _d(Lval))
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return Dval, Lval


def div_impl(S, Dval, Lval, d, diag: int, C, vec: bool = False):
    """Natural-factorization solve in place on C (n x nrhs, Fortran order,
    elimination order)."""
    L = lib()
    C = np.asfortranarray(C, dtype=np.float64)
    if C.ndim == 1:
        C2 = C.reshape(-1, 1, order="F")
    else:
        C2 = C
    nrhs = C2.shape[1]
    rc = L.mfo_div_impl(S.n, S.nfr, _p(S.resptr), _p(S.sepptr), _p(S.reltgt), _p(S.chdptr), _p(S.chdtgt),
                        _p(S.Dptr), _p(S.Lptr), S.nMptr, S.nNval, S.nFval, diag, _d(Dval), _d(Lval), _d(d),
                        _d(C2), nrhs, S.n, 1 if vec else 0)
    if rc != 0:
        raise MemoryError("oracle allocation failed")
    return C


class OracleSymbolic:
    """The fields of a ChordalSymbolic (chordal_symbolic.jl:15-28), 0-based,
    as the oracle's own symbolic analysis computes them."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def ndz(self):
        return int(self.Dptr[-1])

    @property
    def nlz(self):
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

    def factor_flops(self):
        nn = np.diff(self.resptr).astype(np.float64)
        na = np.diff(self.sepptr).astype(np.float64)
        return float(np.sum(nn ** 3 / 3.0 + nn * nn * na + nn * na * na))


class OraclePermutation:
    def __init__(self, perm):
        self.perm = np.ascontiguousarray(perm, dtype=np.int64)
        self.invp = np.empty_like(self.perm)
        self.invp[self.perm] = np.arange(self.perm.size, dtype=np.int64)


def _csc(A):
    import scipy.sparse as sp
    C = sp.csc_matrix(A if sp.issparse(A) else np.asarray(A, dtype=np.float64))
    C.sum_duplicates()
    C.sort_indices()
    return C


def pattern(A):
    """(colptr, rowval) of the symmetric pattern of A, rows ascending (the
    adjacency lists the reference reads from a SparseMatrixCSC)."""
    C = _csc(A)
    C.data = np.ones_like(C.data)
    P = (C + C.T).tocsc()
    P.sort_indices()
    return P.indptr.astype(np.int64), P.indices.astype(np.int64)


def grid_nd_order(nx, ny, nz=1, leaf=8):
    """Nested-dissection order of an nx x ny x nz grid by recursive coordinate
    bisection (vertex id x + nx*(y + ny*z)): the explicit permutation the
    3D benchmark workloads pass to symbolic (the reference accepts an order
    vector, elimination_algorithms.jl:776-779).  Boxes of at most `leaf`
    vertices (or at most 2 along every axis) are numbered x fastest; a larger
    box is split at the middle plane of its longest axis (x, then y, then z on
    ties), and numbered first half, second half, then the separator plane x
    fastest."""
    out = []

    def plain(x0, x1, y0, y1, z0, z1):
        z, y, x = np.meshgrid(np.arange(z0, z1), np.arange(y0, y1), np.arange(x0, x1), indexing="ij")
        out.append((x + nx * (y + ny * z)).ravel())

    def box(x0, x1, y0, y1, z0, z1):
        sx, sy, sz = x1 - x0, y1 - y0, z1 - z0
        if sx <= 0 or sy <= 0 or sz <= 0:
            return
        if sx * sy * sz <= leaf or (sx <= 2 and sy <= 2 and sz <= 2):
            plain(x0, x1, y0, y1, z0, z1)
            return
        if sx >= sy and sx >= sz:
            m = x0 + sx // 2
            box(x0, m, y0, y1, z0, z1); box(m + 1, x1, y0, y1, z0, z1); plain(m, m + 1, y0, y1, z0, z1)
        elif sy >= sz:
            m = y0 + sy // 2
            box(x0, x1, y0, m, z0, z1); box(x0, x1, m + 1, y1, z0, z1); plain(x0, x1, m, m + 1, z0, z1)
        else:
            m = z0 + sz // 2
            box(x0, x1, y0, y1, z0, m); box(x0, x1, y0, y1, m + 1, z1); plain(x0, x1, y0, y1, m, m + 1)

    box(0, nx, 0, ny, 0, nz)
    return np.concatenate(out).astype(np.int64)


def amf_order(A):
    """The reference's default AMF() order (order[k] = vertex eliminated k-th)."""
    colptr, rowval = pattern(A)
    n = colptr.size - 1
    order = np.empty(n, np.int64)
    rc = lib().mfo_amf_order(n, _p(colptr), _p(rowval), _p(order))
    if rc != 0:
        raise RuntimeError(f"mfo_amf_order failed ({rc})")
    return order


def symbolic(A, alg="amf"):
    """(permutation, symbolic factorization) of A under AMF ("amf") or an
    explicit order vector, with Maximal supernodes (symbolic(A; alg),
    chordal_symbolic.jl:68-91)."""
    colptr, rowval = pattern(A)
    n = colptr.size - 1
    order = amf_order(A) if isinstance(alg, str) and alg == "amf" else np.ascontiguousarray(alg, dtype=np.int64)
    L = lib()
    h = L.mfo_symbolic_create(n, _p(colptr), _p(rowval), _p(order))
    if not h:
        raise RuntimeError("mfo_symbolic_create failed")
    try:
        sz = np.zeros(7, np.int64)
        L.mfo_symbolic_sizes(h, _p(sz))
        nfr, nsep = int(sz[1]), int(sz[2])
        a = {k: np.empty(m, np.int64) for k, m in
             [("perm", n), ("resptr", nfr + 1), ("sepptr", nfr + 1), ("septgt", nsep), ("reltgt", nsep),
              ("pnt", nfr), ("chdptr", nfr + 2), ("chdtgt", nfr), ("idx", n), ("Dptr", nfr + 1), ("Lptr", nfr + 1)]}
        L.mfo_symbolic_arrays(h, *[_p(a[k]) for k in ["perm", "resptr", "sepptr", "septgt", "reltgt", "pnt",
                                                       "chdptr", "chdtgt", "idx", "Dptr", "Lptr"]])
    finally:
        L.mfo_symbolic_free(h)
    perm = a.pop("perm")
    S = OracleSymbolic(n=n, nfr=nfr, nMptr=int(sz[3]), nMval=int(sz[4]), nNval=int(sz[5]), nFval=int(sz[6]), **a)
    return OraclePermutation(perm), S


def lower_values(A):
    """Stored entries of the lower triangle of symmetric A, column by column,
    rows ascending (the values Hermitian(A, :L) holds)."""
    import scipy.sparse as sp
    return sp.tril(_csc(A), format="csc")


def assemble(S, invp, A):
    """Dval/Lval holding the permuted lower triangle of A: copyto!(F, A) =
    sympermute (utils.jl:147-219) + copyto!(::ChordalTriangular, ...)
    (chordal_triangular.jl:852-893).  Returns (Dval, Lval, lower triangle of
    A, slot) with slot[k] the flat [Dval; Lval] index of its k-th entry."""
    Lo = lower_values(A)
    Lo.sort_indices()
    n = Lo.shape[0]
    cols = np.repeat(np.arange(n, dtype=np.int64), np.diff(Lo.indptr))
    rows = Lo.indices.astype(np.int64)
    pi, pj = invp[rows], invp[cols]
    r = np.maximum(pi, pj)
    c = np.minimum(pi, pj)
    f = S.idx[c]
    r0 = S.resptr[f]
    r1 = S.resptr[f + 1]
    nn = r1 - r0
    na = S.sepptr[f + 1] - S.sepptr[f]
    slot = np.empty(r.size, np.int64)
    inD = r < r1
    slot[inD] = S.Dptr[f[inD]] + (r[inD] - r0[inD]) + (c[inD] - r0[inD]) * nn[inD]
    off = ~inD
    if np.any(off):
        big = np.int64(n + 1)
        keys = np.repeat(np.arange(S.nfr, dtype=np.int64), np.diff(S.sepptr)) * big + S.septgt
        want = f[off] * big + r[off]
        loc = np.searchsorted(keys, want)
        if np.any(loc >= keys.size) or np.any(keys[np.minimum(loc, keys.size - 1)] != want):
            raise ValueError("matrix entry outside the symbolic pattern")
        slot[off] = S.ndz + S.Lptr[f[off]] + (loc - S.sepptr[f[off]]) + (c[off] - r0[off]) * na[off]
    flat = np.zeros(S.ndz + S.nlz, np.float64)
    flat[slot] = Lo.data
    return flat[:S.ndz].copy(), flat[S.ndz:].copy(), Lo, slot


def factor_and_solve(A, P, S, B, diag: int = 0, signs=None):
    """Oracle x = A^{-1} B (original order) -- ldiv!! (divide.jl:1762-1764)."""
    Dval, Lval, _, _ = assemble(S, P.invp, A)
    info, Dval, Lval, d = chol_impl(S, Dval, Lval, diag, signs)
    if info != 0:
        return info, None, (Dval, Lval, d)
    B = np.asarray(B, dtype=np.float64)
    vec = B.ndim == 1
    C = np.asfortranarray(B[P.perm] if vec else B[P.perm, :])
    C = div_impl(S, Dval, Lval, d, diag, C, vec=vec)
    X = np.empty_like(C)
    if vec:
        X[P.perm] = C
    else:
        X[P.perm, :] = C
    return 0, X, (Dval, Lval, d)
