"""ctypes bindings for the two native libraries of this package.

``libctsym.so``  host-only symbolic analysis (C++, include/cliquetrees_symbolic.h)
``libmfgpu.so``  CUDA sm_100a numeric phase (include/mfgpu.h)

Both are built in-tree by ``build.py``; nothing here falls back to another
implementation when a library is missing -- the import error is raised.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))

_i64 = ctypes.c_int64
_p64 = ctypes.POINTER(ctypes.c_int64)
_pd = ctypes.POINTER(ctypes.c_double)
_pf = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


class NativeLibraryMissing(ImportError):
    pass


def _load(name: str) -> ctypes.CDLL:
    path = os.path.join(_HERE, name)
    if not os.path.exists(path):
        raise NativeLibraryMissing(
            f"{name} is not built ({path}); run `python cliquetrees.jl_b200/build.py`")
    return ctypes.CDLL(path)


_sym = None
_gpu = None


def symlib() -> ctypes.CDLL:
    global _sym
    if _sym is None:
        lib = _load("libctsym.so")
        lib.ct_symbolic_create.argtypes = [_i64, _p64, _p64, _p64, ctypes.POINTER(_vp)]
        lib.ct_symbolic_create.restype = ctypes.c_int
        lib.ct_symbolic_destroy.argtypes = [_vp]
        lib.ct_symbolic_destroy.restype = None
        lib.ct_symbolic_sizes.argtypes = [_vp, _p64]
        lib.ct_symbolic_sizes.restype = ctypes.c_int
        lib.ct_symbolic_arrays.argtypes = [_vp] + [_p64] * 12
        lib.ct_symbolic_arrays.restype = ctypes.c_int
        lib.ct_grid_nd_order.argtypes = [_i64, _i64, _i64, _i64, _p64]
        lib.ct_grid_nd_order.restype = ctypes.c_int
        lib.ct_mindeg_order.argtypes = [_i64, _p64, _p64, _p64]
        lib.ct_mindeg_order.restype = ctypes.c_int
        lib.ct_amf_order.argtypes = [_i64, _p64, _p64, _p64]
        lib.ct_amf_order.restype = ctypes.c_int
        lib.ct_last_error.argtypes = []
        lib.ct_last_error.restype = ctypes.c_char_p
        _sym = lib
    return _sym


def gpulib() -> ctypes.CDLL:
    """The CUDA library.  Raises if it is not built; there is no fallback."""
    global _gpu
    if _gpu is None:
        lib = _load("libmfgpu.so")
        pp = ctypes.POINTER(_vp)
        lib.mf_create.argtypes = [_i64, _i64] + [_p64] * 8 + [ctypes.c_int, ctypes.c_int, ctypes.c_int, pp]
        lib.mf_create.restype = ctypes.c_int
        lib.mf_destroy.argtypes = [_vp]
        lib.mf_destroy.restype = None
        lib.mf_set_stream.argtypes = [_vp, _vp]
        lib.mf_set_stream.restype = ctypes.c_int
        lib.mf_chol_impl.argtypes = [_vp, _pd, _pd, _pd, _pd, _p64]
        lib.mf_chol_impl.restype = ctypes.c_int
        lib.mf_div_impl.argtypes = [_vp, _pd, _i64, _i64]
        lib.mf_div_impl.restype = ctypes.c_int
        lib.mf_set_assembly.argtypes = [_vp, _i64, _p64]
        lib.mf_set_assembly.restype = ctypes.c_int
        lib.mf_assemble.argtypes = [_vp, _pd]
        lib.mf_assemble.restype = ctypes.c_int
        lib.mf_assemble_device.argtypes = [_vp, _vp]
        lib.mf_assemble_device.restype = ctypes.c_int
        lib.mf_factorize.argtypes = [_vp, _pd, _p64]
        lib.mf_factorize.restype = ctypes.c_int
        lib.mf_solve.argtypes = [_vp, _pd, _i64, _i64, _p64]
        lib.mf_solve.restype = ctypes.c_int
        lib.mf_solve_device.argtypes = [_vp, _vp, _i64, _i64, _vp]
        lib.mf_solve_device.restype = ctypes.c_int
        lib.mf_get_factor.argtypes = [_vp, _pd, _pd, _pd]
        lib.mf_get_factor.restype = ctypes.c_int
        lib.mf_synchronize.argtypes = [_vp]
        lib.mf_synchronize.restype = ctypes.c_int
        lib.mf_info.argtypes = [_vp, _p64]
        lib.mf_info.restype = ctypes.c_int
        lib.mf_profile.argtypes = [_vp, ctypes.c_int]
        lib.mf_profile.restype = ctypes.c_int
        lib.mf_kernel_times.argtypes = [_vp, _pd, _p64]
        lib.mf_set_regularization.argtypes = [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        lib.mf_set_regularization.restype = ctypes.c_int
        lib.mf_selinv.argtypes = [_vp]
        lib.mf_selinv.restype = ctypes.c_int
        lib.mf_rescued.argtypes = [_vp, _p64]
        lib.mf_rescued.restype = ctypes.c_int
        lib.mf_logdet.argtypes = [_vp, _pd, _pd]
        lib.mf_logdet.restype = ctypes.c_int
        lib.mf_exec_parents.argtypes = [_vp, _p64]
        lib.mf_exec_parents.restype = ctypes.c_int
        lib.mf_kernel_times.restype = ctypes.c_int
        pint = ctypes.POINTER(ctypes.c_int)
        lib.mf_enable_mixed.argtypes = [_vp]
        lib.mf_enable_mixed.restype = ctypes.c_int
        lib.mf_factorize_mixed.argtypes = [_vp, _pd, _p64, pint]
        lib.mf_factorize_mixed.restype = ctypes.c_int
        lib.mf_solve_refined.argtypes = [_vp, _pd, _i64, _i64, _p64, ctypes.c_double, ctypes.c_int, pint, _pd]
        lib.mf_solve_refined.restype = ctypes.c_int
        lib.mf_solve_refined_device.argtypes = [_vp, _vp, _i64, _i64, _vp, ctypes.c_double, ctypes.c_int, pint,
                                                _pd]
        lib.mf_solve_refined_device.restype = ctypes.c_int
        lib.mf_get_factor_mixed.argtypes = [_vp, _pd, _pd, _pd, _pd]
        lib.mf_get_factor_mixed.restype = ctypes.c_int
        lib.mf_exec_sizes.argtypes = [_vp, _p64, _p64]
        lib.mf_exec_sizes.restype = ctypes.c_int
        lib.mf_plan_info.argtypes = [_i64, _i64] + [_p64] * 8 + [ctypes.c_int, _p64]
        lib.mf_plan_info.restype = ctypes.c_int
        lib.mf_set_segments.argtypes = [_vp, _i64, _p64]
        lib.mf_set_segments.restype = ctypes.c_int
        lib.mf_segment_errors.argtypes = [_vp, _pd]
        lib.mf_segment_errors.restype = ctypes.c_int
        lib.mf_autotune.argtypes = [_vp, ctypes.c_int, _pd]
        lib.mf_autotune.restype = ctypes.c_int
        p32 = ctypes.POINTER(ctypes.c_int32)
        lib.mf_kernel_choice.argtypes = [_vp, p32, p32]
        lib.mf_kernel_choice.restype = ctypes.c_int
        lib.mf_set_kernel_choice.argtypes = [_vp, p32, p32]
        lib.mf_set_kernel_choice.restype = ctypes.c_int
        lib.mf_last_error.argtypes = []
        lib.mf_last_error.restype = ctypes.c_char_p
        _gpu = lib
    return _gpu


class MFError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc != 0:
        msg = gpulib().mf_last_error().decode(errors="replace")
        raise MFError(f"{what} failed ({rc}): {msg}")


def ptr64(a):
    """int64 numpy array -> ctypes pointer (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(_p64)


def ptrd(a):
    if a is None:
        return None
    return a.ctypes.data_as(_pd)


def ptrf(a):
    if a is None:
        return None
    return a.ctypes.data_as(_pf)
