"""Build the native libraries of this package in-tree.

  multifrontal/libctsym.so  host symbolic analysis (g++)
  multifrontal/libmfgpu.so  CUDA sm_100a numeric phase (nvcc)

Usage: python cliquetrees.jl_b200/build.py [--only sym|gpu] [--verbose]
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "multifrontal")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

GPU_SOURCES = ["mf_plan.cu", "mf_factor.cu", "mf_tc.cu", "mf_solve.cu", "mf_refine.cu", "mf_api.cu", "mf_static.cu",
               "mf_selinv.cu"]
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_sym(verbose=False, force=False):
    src = [os.path.join(CSRC, "symbolic.cpp"), os.path.join(CSRC, "mindeg.cpp"), os.path.join(CSRC, "amf.cpp")]
    hdr = [os.path.join(HERE, "..", "include", "cliquetrees_symbolic.h")]
    target = os.path.join(OUT, "libctsym.so")
    if force or _stale(target, src + hdr):
        # -ffp-contract=off: the AMF fill score must round exactly as the reference's
        # separate multiply and subtract do
        _run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-Wall", "-o", target] + src,
             verbose)
    return target


def build_gpu(verbose=False, force=False, ptxas_verbose=False):
    src = [os.path.join(CSRC, s) for s in GPU_SOURCES]
    hdr = [os.path.join(CSRC, "mf_internal.cuh"), os.path.join(HERE, "..", "include", "mfgpu.h")]
    target = os.path.join(OUT, "libmfgpu.so")
    if force or _stale(target, src + hdr):
        cmd = [NVCC, "-O3", "-std=c++17", "-lineinfo", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
               "--expt-relaxed-constexpr"] + GENCODE + ["-o", target] + src + [
                   "-lcublas", "-Xlinker", "-rpath," + os.path.join(os.path.dirname(os.path.dirname(NVCC)), "lib64")]
        if ptxas_verbose:
            cmd.insert(1, "-Xptxas=-v")
        _run(cmd, verbose)
    return target


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", choices=["sym", "gpu"], default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args(argv)
    if a.only in (None, "sym"):
        print(build_sym(a.verbose, a.force))
    if a.only in (None, "gpu"):
        print(build_gpu(a.verbose, a.force, a.ptxas))


if __name__ == "__main__":
    sys.exit(main())
