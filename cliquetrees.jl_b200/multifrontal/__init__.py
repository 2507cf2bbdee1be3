"""B200-native numeric phase of CliqueTrees.jl's Multifrontal submodule.

Host mirror of the reference API (src/Multifrontal.jl/src/Multifrontal.jl:25-33
exports): symbolic analysis on the host (C++), Cholesky / LDLt factorization
and supernodal solves on the GPU (CUDA sm_100a, ``libmfgpu.so``).
"""
from .symbolic import ChordalSymbolic, Permutation, symbolic, grid_nd_order, amf_order, mindeg_order
from .factorization import (ChordalFactorization, ChordalCholesky, ChordalLDLt, PosDefException,
                            SingularException, cholesky_, ldlt_, ldiv, rdiv, issuccess, logdet, logabsdet, det,
                            chol_impl, selinv_, NoRegularization, DynamicRegularization)
from . import testmatrices

__all__ = [
    "ChordalSymbolic", "Permutation", "symbolic", "grid_nd_order", "amf_order", "mindeg_order",
    "ChordalFactorization", "ChordalCholesky", "ChordalLDLt", "PosDefException", "SingularException",
    "cholesky_", "ldlt_", "ldiv", "rdiv", "issuccess", "logdet", "logabsdet", "det", "chol_impl", "selinv_", "NoRegularization",
    "DynamicRegularization", "testmatrices",
]
