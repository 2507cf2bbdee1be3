"""Factorization objects and the numeric entry points, mirroring the
reference's Julia API for the multifrontal hot path.

  ChordalCholesky(A; alg) / ChordalLDLt(A; alg)
        src/Multifrontal.jl/src/chordal_factorization.jl:1-20, :45, :95, :146-239
  cholesky_(F; check)   = cholesky!(F)     src/Multifrontal.jl/src/cholesky.jl:80-101
  ldlt_(F; signs, check) = ldlt!(F)        src/Multifrontal.jl/src/cholesky.jl:181-203
  factorize! info mapping (info -> perm[info])  cholesky.jl:233-257
  checkinfo (PosDefException / SingularException)  utils.jl:775-785
  ldiv(F, B)  = F \\ B = ldiv!!            src/Multifrontal.jl/src/divide.jl:201-206, :1762-1764
  rdiv(B, F)  = B / F = rdiv!!             src/Multifrontal.jl/src/divide.jl:287-292, :1769-1771
  issuccess, logdet, det                   abstract_factorization.jl:100-102, :156-179
  flatindices / value refresh              chordal_symbolic.jl:731-752, chordal_factorization.jl:322-338

Every numeric operation runs in ``libmfgpu.so`` on the GPU; there is no CPU
code path for the numbers.  Python ``!`` cannot appear in names, so
``cholesky!`` is ``cholesky_`` and ``ldlt!`` is ``ldlt_``.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native
from ._native import check, ptr64, ptrd
from .sparse import assembly_map
from .symbolic import ChordalSymbolic, Permutation, symbolic


class PosDefException(Exception):
    """LinearAlgebra.PosDefException(info): pivot `info` (1-based, original order) was not positive."""

    def __init__(self, info):
        super().__init__(f"matrix is not positive definite; pivot {info} failed")
        self.info = info


class SingularException(Exception):
    """LinearAlgebra.SingularException(info): pivot `info` (1-based, original order) is zero."""

    def __init__(self, info):
        super().__init__(f"matrix is singular; pivot {info} is zero")
        self.info = info


class _Handle:
    """Owns one device handle (pattern + factor)."""

    def __init__(self, S: ChordalSymbolic, diag: int, nrhs_cap: int, device: int):
        lib = _native.gpulib()
        h = ctypes.c_void_p()
        rc = lib.mf_create(S.n, S.nfr, ptr64(S.resptr), ptr64(S.sepptr), ptr64(S.septgt), ptr64(S.reltgt),
                           ptr64(S.chdptr), ptr64(S.chdtgt), ptr64(S.Dptr), ptr64(S.Lptr), diag, nrhs_cap,
                           device, ctypes.byref(h))
        check(rc, "mf_create")
        self.h = h
        self.lib = lib

    def close(self):
        if self.h is not None and self.h.value:
            self.lib.mf_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ChordalFactorization:
    """``ChordalFactorization{DIAG, :L, Float64, Int}`` with its numeric
    storage on the GPU.  ``diag = 0`` is ChordalCholesky (DIAG = :N),
    ``diag = 1`` is ChordalLDLt (DIAG = :U)."""

    DIAG = 0

    def __init__(self, A, P: Permutation | None = None, S: ChordalSymbolic | None = None, *, alg="amf",
                 device: int = 0, nrhs_cap: int = 16, mixed: bool = False, tol: float = 1e-12, maxit: int = 100):
        """``mixed=True`` selects the mixed-precision form: FP32 fronts on the
        GPU, FP64 refinement in ``ldiv`` to backward error ``tol`` (the
        reference has no such mode; see the module docstring)."""
        if (P is None) != (S is None):
            raise ValueError("pass both P and S or neither")
        if P is None:
            P, S = symbolic(A, alg=alg)
        self.P = P
        self.S = S
        self.info = 0
        self.mixed = mixed
        self.tol = tol
        self.maxit = maxit
        self.used_fp64 = False
        self.rescued = 0  # fronts / diagonal blocks the mixed factorization redid in FP64
        self.last_refinement = None
        self._factored = False
        self._handle = _Handle(S, self.DIAG, nrhs_cap, device)
        self._slot_for = None
        self.copyto(A)

    # -- reference fields ------------------------------------------------
    @property
    def perm(self):
        return self.P.perm

    @property
    def invp(self):
        return self.P.invp

    @property
    def n(self):
        return self.S.n

    def copyto(self, A):
        """copyto!(F, A) (abstract_factorization.jl:68-71): assemble A's
        values into the factor storage.  The slot map (flatindices) is
        computed once per pattern and cached on the device."""
        Lo, slot = assembly_map(self.S, self.P.invp, A)
        key = (Lo.indptr.tobytes(), Lo.indices.tobytes())
        lib = self._handle.lib
        if self._slot_for != key:
            slot = np.ascontiguousarray(slot, dtype=np.int64)
            check(lib.mf_set_assembly(self._handle.h, slot.size, ptr64(slot)), "mf_set_assembly")
            self._slot_for = key
            if self.mixed:
                check(lib.mf_enable_mixed(self._handle.h), "mf_enable_mixed")
        vals = np.ascontiguousarray(Lo.data, dtype=np.float64)
        check(lib.mf_assemble(self._handle.h, ptrd(vals)), "mf_assemble")
        self._factored = False
        return self

    def refresh(self, values):
        """Value refresh on the cached pattern: ``values`` are A's stored
        lower-triangle entries in the order of the matrix passed at
        construction (setflatindex! loop, test/multifrontal.jl:76-113)."""
        vals = np.ascontiguousarray(values, dtype=np.float64)
        check(self._handle.lib.mf_assemble(self._handle.h, ptrd(vals)), "mf_assemble")
        self._factored = False
        return self

    def factor_arrays(self):
        """(Dval, Lval, d) in the reference layout, downloaded from the GPU."""
        Dval = np.empty(self.S.ndz, np.float64)
        Lval = np.empty(self.S.nlz, np.float64)
        d = np.ones(self.S.n, np.float64)
        check(self._handle.lib.mf_get_factor(self._handle.h, ptrd(Dval), ptrd(Lval),
                                             ptrd(d) if self.DIAG else None), "mf_get_factor")
        return Dval, Lval, d

    def factor_arrays_mixed(self):
        """(Dval, Lval, d, scale) of the single-precision factor of S A S
        (mixed form only)."""
        Dval = np.empty(self.S.ndz, np.float64)
        Lval = np.empty(self.S.nlz, np.float64)
        d = np.ones(self.S.n, np.float64)
        sc = np.empty(self.S.n, np.float64)
        check(self._handle.lib.mf_get_factor_mixed(self._handle.h, ptrd(Dval), ptrd(Lval),
                                                   ptrd(d) if self.DIAG else None, ptrd(sc)), "mf_get_factor_mixed")
        return Dval, Lval, d, sc

    @property
    def Dval(self):
        return self.factor_arrays()[0]

    @property
    def Lval(self):
        return self.factor_arrays()[1]

    @property
    def d(self):
        return self.factor_arrays()[2]

    # -- numeric phase -----------------------------------------------------
    def _factorize(self, signs, check_info: bool):
        sg = None
        if signs is not None:
            # permuteto(T, signs, F.perm) (cholesky.jl:242)
            sg = np.ascontiguousarray(np.asarray(signs, dtype=np.float64)[self.P.perm])
        info = ctypes.c_int64(0)
        if self.mixed:
            fp64 = ctypes.c_int(0)
            check(self._handle.lib.mf_factorize_mixed(self._handle.h, ptrd(sg), ctypes.byref(info), ctypes.byref(fp64)),
                  "mf_factorize_mixed")
            self.used_fp64 = bool(fp64.value)
            cnt = ctypes.c_int64(0)
            check(self._handle.lib.mf_rescued(self._handle.h, ctypes.byref(cnt)), "mf_rescued")
            self.rescued = int(cnt.value)
        else:
            check(self._handle.lib.mf_factorize(self._handle.h, ptrd(sg), ctypes.byref(info)), "mf_factorize")
        k = int(info.value)
        # factorize! level 1: local info -> perm[info] (cholesky.jl:250-254)
        self.info = 0 if k == 0 else int(self.P.perm[k - 1]) + 1
        self._factored = True
        if check_info and self.info != 0:
            if self.DIAG == 0:
                raise PosDefException(self.info)
            raise SingularException(self.info)
        return self

    def issuccess(self) -> bool:
        return self._factored and self.info == 0

    def autotune(self, reps: int = 3) -> dict:
        """Mixed form only: time every tree level's single-precision GEMM roles
        with the tcgen05 tiles and with the FFMA tiles on the current values
        and keep the faster per level (the factor is then refactored).
        Returns the GEMM-role milliseconds of each choice and the per-level
        picks."""
        if not self.mixed:
            raise ValueError("autotune applies to the mixed form")
        lib, h = self._handle.lib, self._handle.h
        ms = np.zeros(6, np.float64)
        check(lib.mf_autotune(h, int(reps), ptrd(ms)), "mf_autotune")
        nl = int(ms[5])
        tc_steps = np.zeros(nl, np.int32)
        tc_syrk = np.zeros(nl, np.int32)
        p32 = ctypes.POINTER(ctypes.c_int32)
        check(lib.mf_kernel_choice(h, tc_steps.ctypes.data_as(p32), tc_syrk.ctypes.data_as(p32)),
              "mf_kernel_choice")
        self._factored = False
        return {"tc_ms": float(ms[0]), "ffma_ms": float(ms[1]), "tuned_ms": float(ms[2]),
                "tc_steps": tc_steps, "tc_syrk": tc_syrk}

    def set_kernel_choice(self, tc_steps=None, tc_syrk=None):
        """Set the per-level choice (1 = tcgen05, 0 = FFMA) directly, e.g. one
        saved from ``autotune`` on another handle of the same pattern."""
        p32 = ctypes.POINTER(ctypes.c_int32)
        info = np.zeros(9, np.int64)
        check(self._handle.lib.mf_info(self._handle.h, ptr64(info)), "mf_info")
        a = None if tc_steps is None else np.ascontiguousarray(tc_steps, dtype=np.int32)
        b = None if tc_syrk is None else np.ascontiguousarray(tc_syrk, dtype=np.int32)
        for v in (a, b):
            if v is not None and v.size != info[7]:
                raise ValueError(f"kernel choice needs one entry per tree level ({info[7]}), got {v.size}")
        check(self._handle.lib.mf_set_kernel_choice(self._handle.h, None if a is None else a.ctypes.data_as(p32),
                                                    None if b is None else b.ctypes.data_as(p32)),
              "mf_set_kernel_choice")

    def solve(self, B):
        return ldiv(self, B)

    def logabsdet(self):
        """(log|det A|, sign det A), reduced on the GPU from the factor's
        diagonal (logabsdet, abstract_factorization.jl:175-181)."""
        if not self._factored:
            raise RuntimeError("factorize first (cholesky_ / ldlt_)")
        la = ctypes.c_double(0.0)
        sg = ctypes.c_double(0.0)
        check(self._handle.lib.mf_logdet(self._handle.h, ctypes.byref(la), ctypes.byref(sg)), "mf_logdet")
        return float(la.value), float(sg.value)

    def logdet(self) -> float:
        """logdet(F) (abstract_factorization.jl:167-173): 2 logdet(L) for
        Cholesky; log|det| + log(sign) for LDLt, which, as Julia's log of a
        negative number, raises for a negative determinant."""
        la, sg = self.logabsdet()
        if sg < 0:
            raise ValueError("logdet of a matrix with negative determinant (DomainError in the reference)")
        return la if sg > 0 else -np.inf

    def det(self) -> float:
        """det(F) (abstract_factorization.jl:159-165)."""
        la, sg = self.logabsdet()
        return float(sg * np.exp(la))

    def close(self):
        self._handle.close()


class ChordalCholesky(ChordalFactorization):
    """P A P^T = L L^T (chordal_factorization.jl:22-45)."""
    DIAG = 0


class ChordalLDLt(ChordalFactorization):
    """P A P^T = L D L^T with static 1x1 pivots (chordal_factorization.jl:70-95)."""
    DIAG = 1


class NoRegularization:
    """Pivot rule: reject a pivot of the wrong sign (no_regularization.jl:27-42)."""


class DynamicRegularization:
    """Pivot rule: a pivot d_j with s_j d_j < epsilon becomes delta s_j
    (dynamic_regularization.jl:38-90); negative fields take the defaults
    cbrt(eps) and sqrt(eps)."""

    def __init__(self, delta: float = -1.0, epsilon: float = -1.0):
        self.delta = float(delta)
        self.epsilon = float(epsilon)


def _set_reg(F, reg):
    if reg is None or isinstance(reg, NoRegularization):
        check(F._handle.lib.mf_set_regularization(F._handle.h, 0, -1.0, -1.0), "mf_set_regularization")
    elif isinstance(reg, DynamicRegularization):
        if F.mixed:
            raise ValueError("DynamicRegularization applies to the FP64 factorization (mixed=False)")
        check(F._handle.lib.mf_set_regularization(F._handle.h, 1, reg.delta, reg.epsilon), "mf_set_regularization")
    else:
        raise TypeError(f"unsupported regularization {type(reg).__name__}")


def cholesky_(F: ChordalFactorization, *, check: bool = True, reg=None):
    """cholesky!(F; check, reg) (cholesky.jl:80-101): signs = ones."""
    if F.DIAG != 0:
        raise TypeError("cholesky_ needs a ChordalCholesky")
    _set_reg(F, reg)
    return F._factorize(None, check)


def ldlt_(F: ChordalFactorization, *, signs=None, check: bool = True, reg=None):
    """ldlt!(F; signs=zeros, check, reg) (cholesky.jl:181-203)."""
    if F.DIAG != 1:
        raise TypeError("ldlt_ needs a ChordalLDLt")
    _set_reg(F, reg)
    return F._factorize(signs, check)


def ldiv(F: ChordalFactorization, B):
    """F \\ B (divide.jl:201-206): x = P^T L^-T D^-1 L^-1 P b, on the GPU."""
    if not F._factored:
        raise RuntimeError("factorize first (cholesky_ / ldlt_)")
    if F.info != 0:
        raise RuntimeError("factorization failed; no solve possible")
    B = np.asarray(B, dtype=np.float64)
    vec = B.ndim == 1
    X = np.asfortranarray(B.reshape(-1, 1) if vec else B).copy(order="F")
    if X.shape[0] != F.n:
        raise ValueError("dimension mismatch")
    if F.mixed:
        it = ctypes.c_int(0)
        eta = ctypes.c_double(0.0)
        check(F._handle.lib.mf_solve_refined(F._handle.h, ptrd(X), X.shape[1], F.n, ptr64(F.P.perm), F.tol, F.maxit,
                                             ctypes.byref(it), ctypes.byref(eta)), "mf_solve_refined")
        F.last_refinement = (int(it.value), float(eta.value))
    else:
        check(F._handle.lib.mf_solve(F._handle.h, ptrd(X), X.shape[1], F.n, ptr64(F.P.perm)), "mf_solve")
    return X[:, 0].copy() if vec else X


def rdiv(B, F: ChordalFactorization):
    """B / F for a symmetric factorization: (F \\ B^T)^T (divide.jl:287-292)."""
    B = np.asarray(B, dtype=np.float64)
    return ldiv(F, B.T).T


def selinv_(F: ChordalFactorization):
    """selinv!(F) (selinv.jl:38-41): replace the Cholesky factor on the GPU by
    the entries of A^{-1} on the pattern of L (``F.factor_arrays()`` then
    returns them in the reference layout); F must be factorized again before
    a solve."""
    if F.DIAG != 0:
        raise TypeError("selinv_ needs a ChordalCholesky")
    if not F._factored or F.info != 0:
        raise RuntimeError("factorize first (cholesky_)")
    if F.mixed:
        raise ValueError("selinv_ needs the FP64 factor: use a plain (mixed=False) factorization")
    check(F._handle.lib.mf_selinv(F._handle.h), "mf_selinv")
    F._factored = False
    return F


def issuccess(F: ChordalFactorization) -> bool:
    return F.issuccess()


def logdet(F: ChordalFactorization) -> float:
    return F.logdet()


def logabsdet(F: ChordalFactorization):
    return F.logabsdet()


def det(F: ChordalFactorization) -> float:
    return F.det()


# -- the drop-in boundary in the reference's own terms -----------------------

def chol_impl(S: ChordalSymbolic, Dval, Lval, *, diag: int, signs=None, d=None, device: int = 0):
    """chol_impl! (cholesky.jl:361-392) on the GPU through the C ABI:
    Dval/Lval hold the assembled (permuted) matrix and are overwritten with
    the factor; returns (info, d) with info the 1-based permuted column of
    the first rejected pivot (0 on success)."""
    h = _Handle(S, diag, 1, device)
    try:
        Dval = np.ascontiguousarray(Dval, dtype=np.float64)
        Lval = np.ascontiguousarray(Lval, dtype=np.float64)
        if d is None:
            d = np.zeros(S.n, np.float64)
        sg = None if signs is None else np.ascontiguousarray(signs, dtype=np.float64)
        info = ctypes.c_int64(0)
        check(h.lib.mf_chol_impl(h.h, ptrd(Dval), ptrd(Lval), ptrd(d) if diag else None, ptrd(sg),
                                 ctypes.byref(info)), "mf_chol_impl")
        return int(info.value), Dval, Lval, d
    finally:
        h.close()
