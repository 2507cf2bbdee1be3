"""The C-ABI libraries load and export every symbol their headers declare
(no compute calls: runs without a GPU)."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return set(re.findall(r"\b(?:int|void|const char\*)\s+\**(\w+)\s*\(", src))


def test_gpu_library_exports_header_symbols():
    path = os.path.join(ROOT, "cliquetrees.jl_b200", "multifrontal", "libmfgpu.so")
    if not os.path.exists(path):
        import importlib
        importlib.import_module("build").build_gpu()
    lib = ctypes.CDLL(path)
    names = declared("mfgpu.h")
    assert "mf_create" in names and "mf_chol_impl" in names and "mf_div_impl" in names
    for name in names:
        assert hasattr(lib, name), name


def test_symbolic_library_exports_header_symbols():
    path = os.path.join(ROOT, "cliquetrees.jl_b200", "multifrontal", "libctsym.so")
    lib = ctypes.CDLL(path)
    for name in declared("cliquetrees_symbolic.h"):
        assert hasattr(lib, name), name


def test_gpu_library_without_device_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        return
    import multifrontal as mf
    from multifrontal import testmatrices as tm
    A = tm.grid_laplacian(4, 4)
    try:
        mf.ChordalCholesky(A, alg=mf.grid_nd_order(4, 4, 1))
    except mf.factorization._native.MFError as e:
        assert "no CUDA device" in str(e)
    else:
        raise AssertionError("expected an error without a GPU")
