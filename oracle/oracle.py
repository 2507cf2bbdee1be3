"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for the multifrontal numeric phase.

Python driver around ``mf_oracle.c`` (a C restatement of CliqueTrees.jl's
chol_impl!/div_impl!, see the header of that file for the line-by-line
citations).  Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module; the product never does.

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

_i64 = ctypes.c_int64
_p64 = ctypes.POINTER(ctypes.c_int64)
_pd = ctypes.POINTER(ctypes.c_double)


def build(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.run(["gcc", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-o", LIB, SRC, "-ldl", "-lm"],
                       check=True)
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


def chol_impl(S, Dval, Lval, diag: int, signs=None, d=None):
    """Run the oracle factorization in place.  Returns (info, d)."""
    L = lib()
    Dval = np.ascontiguousarray(Dval, dtype=np.float64)
    Lval = np.ascontiguousarray(Lval, dtype=np.float64)
    if d is None:
        d = np.zeros(max(S.n, 1), np.float64)
    sg = None if signs is None else np.ascontiguousarray(signs, dtype=np.float64)
    info = L.mfo_chol_impl(S.n, S.nfr, _p(S.resptr), _p(S.sepptr), _p(S.reltgt), _p(S.chdptr), _p(S.chdtgt),
                           _p(S.Dptr), _p(S.Lptr), S.nMptr, S.nMval, S.nFval, diag, _d(Dval), _d(Lval), _d(d),
                           _d(sg))
    if info < 0:
        raise MemoryError("oracle allocation failed")
    return int(info), Dval, Lval, d


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


def assemble(S, invp, A):
    """Dval/Lval holding the permuted lower triangle of A (copyto!,
    chordal_triangular.jl:852-893) plus the flat slot map."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "..", "cliquetrees.jl_b200"))
    from multifrontal.sparse import assembly_map
    Lo, slot = assembly_map(S, invp, A)
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
