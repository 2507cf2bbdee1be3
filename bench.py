"""Benchmark: factor + solve of the 80^3 3D 7-point problem on the GPU.

One step = assemble the matrix values on the device, multifrontal Cholesky
factorization, and a 4-right-hand-side solve (permutation included), the
hot path of CliqueTrees.jl's Multifrontal numeric phase
(chol_impl!, cholesky.jl:361-392; ldiv!!, divide.jl:1762-1764).

Workload: 3D 7-point Laplacian on an 80^3 grid (n = 512,000), seeded
log-uniform [1e-3, 1e3] edge coefficients, diagonal = row sum + 1e-6,
geometric nested-dissection order, 4 N(0,1) right-hand sides; synthetic,
the inputs (factor 3.4 GB) are far larger than L2.

value      : solves/s (one solve = factor + 4-RHS solve of one system) with
             the matrix values and right-hand sides already in HBM;
e2e        : the same through the public C ABI with pinned host buffers
             (values + RHS copied in, solution copied out every step);
roofline   : the dominant kernel (per-kernel CUDA events in a separate
             profiling pass) against a DGEMM peak measured in this run;
cpu_baseline: the CPU oracle (C restatement of the reference path, scipy's
             OpenBLAS, all host threads) on one full step.

--impl reference times that CPU path alone (rank 0 only).
Multi-GPU: every rank factors its own replica (no collective); value is
the sum over ranks, time is the max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cliquetrees.jl_b200"))

KERNEL_NAMES = ["assemble", "small", "extend_add", "panel", "update", "syrk", "solve_small", "solve_gather",
                "solve_fwd", "solve_bwd_l", "solve_bwd", "permute", "other", "diag", "left", "residual"]
NK = len(KERNEL_NAMES)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--side", type=int, default=80)
    ap.add_argument("--nrhs", type=int, default=4)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-only", action="store_true")
    ap.add_argument("--mixed-profile", action="store_true", help="with --profile-only: the mixed form")
    return ap.parse_args()


def workload(side, nrhs, seed=2):
    import multifrontal as mf
    from multifrontal import testmatrices as tm
    A = tm.config2(side, seed=seed)
    order = mf.grid_nd_order(side, side, side, 8)
    P, S = mf.symbolic(A, alg=order)
    B = tm.rhs(A.shape[0], nrhs, seed=seed + 1)
    return A, P, S, B


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            self.path = f"/tmp/clocks_{os.getpid()}.csv"
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], 0.0, set()
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 7:
                continue
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except ValueError:
                continue
            for name, v in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"],
                               f[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


def dgemm_peak_tflops(torch, dev):
    """cuBLAS DGEMM 8192^3, best of 5 (the FP64 denominator; MEASURED_PEAKS
    holds only bf16 and copy numbers)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def exec_sizes(lib, h):
    info = np.zeros(9, np.int64)
    lib.mf_info(h, info.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    nex = int(info[8])
    nn = np.zeros(nex, np.int64)
    na = np.zeros(nex, np.int64)
    p64 = ctypes.POINTER(ctypes.c_int64)
    lib.mf_exec_sizes(h, nn.ctypes.data_as(p64), na.ctypes.data_as(p64))
    return nn, na


def kernel_flops(nn, na):
    """Flops per kernel class for one factorization, counted on the fronts
    the device executes (after amalgamation): fronts with nj <= 96 run in
    the fused small kernel; for the others the panel kernels (diagonal
    blocks, TRSM, left and trailing updates) do nn^3/3 + nn^2*na and the
    SYRK kernel nn*na^2."""
    nn = nn.astype(np.float64)
    na = na.astype(np.float64)
    big = (nn + na) > 96
    return {
        "small": float(np.sum((nn ** 3 / 3 + nn * nn * na + nn * na * na)[~big])),
        "panel+update": float(np.sum((nn ** 3 / 3 + nn * nn * na)[big])),
        "syrk": float(np.sum((nn * na * na)[big])),
    }


def cpu_reference_step(A, P, S, B):
    from oracle import oracle
    t0 = time.perf_counter()
    info, X, _ = oracle.factor_and_solve(A, P, S, B, 0)
    dt = time.perf_counter() - t0
    return dt, info, X


def run_reference(args, rank):
    if rank != 0:
        return
    from oracle import oracle
    threads = os.cpu_count() or 1
    oracle.set_threads(threads)
    A, P, S, B = workload(args.side, args.nrhs)
    for _ in range(args.warmup):
        cpu_reference_step(A, P, S, B)
    times = []
    for _ in range(args.steps):
        dt, info, X = cpu_reference_step(A, P, S, B)
        times.append(dt)
    tot = sum(times)
    value = args.steps / tot
    from multifrontal import testmatrices as tm
    eta = float(tm.backward_error(A, X, B).max())
    line = {
        "impl": "reference", "metric": "solves_per_s", "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3d7pt_{args.side}^3_chol_factor+solve_{args.nrhs}rhs", "n": int(S.n),
                   "factor_gflop": S.factor_flops() / 1e9, "ordering": "geometric nested dissection"},
        "backward_error": eta,
        "p50_ms": float(np.percentile(times, 50) * 1e3), "p99_ms": float(np.percentile(times, 99) * 1e3),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": "port",
                         "sample": f"full factor+solve of the {args.side}^3 system per step"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
    if args.impl == "reference":
        run_reference(args, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    import multifrontal as mf
    from multifrontal import _native

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    A, P, S, B = workload(args.side, args.nrhs)

    if args.profile_only:
        r = run_form(args, A, P, S, B, mixed=args.mixed_profile, local=local, world=world, profile_only=True)
        print(json.dumps(r))
        return

    mixed = run_form(args, A, P, S, B, mixed=True, local=local, world=world)
    plain = run_form(args, A, P, S, B, mixed=False, local=local, world=world)

    # roofline: the dominant kernel class of the headline (mixed) form
    peaks = measured_peaks()
    dgemm = dgemm_peak_tflops(torch, dev)
    sgemm = sgemm_peak_tflops(torch, dev)

    def roofline(form, peak, peak_src, fl):
        kt = form["kernels"]
        classes = {
            "syrk": (fl["syrk"], ["syrk"]),
            "panel+update": (fl["panel+update"], ["panel", "update", "diag", "left"]),
            "small": (fl["small"], ["small"]),
        }
        cls_ms = {k: sum(kt[x]["ms"] for x in v[1]) for k, v in classes.items()}
        dom = max(cls_ms, key=cls_ms.get)
        launches = sum(kt[x]["launches"] for x in classes[dom][1])
        kms = cls_ms[dom]
        achieved = classes[dom][0] / (kms / 1e3) / 1e12 if kms > 0 else 0.0
        per_class = {k: {"tflops": classes[k][0] / (cls_ms[k] / 1e3) / 1e12 if cls_ms[k] > 0 else None,
                         "ms": cls_ms[k], "gflop": classes[k][0] / 1e9} for k in classes}
        return {"kernel": dom, "bound": "tensor" if dom != "small" else "latency", "achieved": achieved,
                "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak if peak else None, "traffic": None,
                "peak_source": peak_src, "flops_per_launch": classes[dom][0] / max(launches, 1),
                "avg_launch_ms": kms / max(launches, 1), "classes": per_class}

    roof_mixed = roofline(mixed, sgemm, "cuBLAS SGEMM 8192^3 (FP32, TF32 off) measured in this run", mixed["flops"])
    roof_plain = roofline(plain, dgemm, "cuBLAS DGEMM 8192^3 measured in this run (no FP64 figure in "
                                        "MEASURED_PEAKS.json)", plain["flops"])

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle
        threads = os.cpu_count() or 1
        oracle.set_threads(threads)
        dt, cinfo, _ = cpu_reference_step(A, P, S, B)
        cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": threads, "kind": "port",
               "sample": f"one full FP64 factor+{args.nrhs}-RHS solve of the {args.side}^3 system ({dt:.2f} s)"}

    if rank == 0:
        line = {
            "metric": "solves_per_s", "value": mixed["value"], "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": mixed["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"3d7pt_{args.side}^3_chol_factor+solve_{args.nrhs}rhs", "n": int(S.n),
                       "fronts": int(S.nfr), "factor_gflop": S.factor_flops() / 1e9, "nnz_L": int(S.nnz()),
                       "mode": "mixed: FP32 fronts + FP64 PCG to backward error 1e-12",
                       "l2": "inputs larger than L2 (factor 2-4 GB)", "parallelism": f"replicas x{world}"},
            "p50_ms": mixed["p50_ms"], "p99_ms": mixed["p99_ms"], "backward_error": mixed["backward_error"],
            "refine_iterations": mixed["iterations"],
            "e2e": mixed["e2e"],
            "gpu_launches": mixed["gpu_launches"],
            "roofline": roof_mixed,
            "kernels": mixed["kernels"],
            "clocks": mixed["clocks"],
            "plain_fp64": {"value": plain["value"], "ms_per_step": plain["ms_per_step"],
                           "p50_ms": plain["p50_ms"], "p99_ms": plain["p99_ms"],
                           "backward_error": plain["backward_error"], "e2e": plain["e2e"],
                           "roofline": roof_plain, "kernels": plain["kernels"], "clocks": plain["clocks"]},
            "mixed_over_plain": mixed["value"] / plain["value"],
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def sgemm_peak_tflops(torch, dev):
    """cuBLAS SGEMM 8192^3 with TF32 disabled, best of 5 (the FP32 denominator)."""
    keep = torch.backends.cuda.matmul.allow_tf32
    torch.backends.cuda.matmul.allow_tf32 = False
    n = 8192
    a = torch.randn(n, n, dtype=torch.float32, device=dev)
    b = torch.randn(n, n, dtype=torch.float32, device=dev)
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e9
    for _ in range(5):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    torch.backends.cuda.matmul.allow_tf32 = keep
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def run_form(args, A, P, S, B, *, mixed, local, world, profile_only=False):
    """Time one form (mixed or plain FP64) of the step; returns a dict."""
    import torch
    import multifrontal as mf
    from multifrontal import _native
    from multifrontal import testmatrices as tm
    from multifrontal.sparse import assembly_map

    dev = torch.device("cuda", local)
    n = S.n
    F = mf.ChordalCholesky(A, P, S, device=local, nrhs_cap=16, mixed=mixed)
    lib = _native.gpulib()
    h = F._handle.h
    stream = torch.cuda.Stream(device=dev)
    _native.check(lib.mf_set_stream(h, ctypes.c_void_p(stream.cuda_stream)), "mf_set_stream")
    Lo, _ = assembly_map(S, P.invp, A)
    nz_host = torch.from_numpy(np.ascontiguousarray(Lo.data)).pin_memory()
    nz_dev = nz_host.to(dev)
    B_host = torch.from_numpy(np.asfortranarray(B).ravel(order="F").copy()).pin_memory()
    B_dev0 = B_host.to(dev)
    X_dev = torch.empty_like(B_dev0)
    perm_dev = torch.from_numpy(P.perm.astype(np.int64)).to(dev)
    X_host = torch.empty_like(B_host).pin_memory()
    info = ctypes.c_int64(0)
    fp64 = ctypes.c_int(0)
    iters = ctypes.c_int(0)
    eta_dev = ctypes.c_double(0.0)
    vp = ctypes.c_void_p
    pd = ctypes.POINTER(ctypes.c_double)
    tol, maxit = 1e-12, 100

    def step_device():
        # the RHS copy must run on the library's stream (same stream order)
        with torch.cuda.stream(stream):
            X_dev.copy_(B_dev0)
        _native.check(lib.mf_assemble_device(h, vp(nz_dev.data_ptr())), "assemble")
        if mixed:
            _native.check(lib.mf_factorize_mixed(h, None, ctypes.byref(info), ctypes.byref(fp64)), "factorize")
            _native.check(lib.mf_solve_refined_device(h, vp(X_dev.data_ptr()), args.nrhs, n, vp(perm_dev.data_ptr()),
                                                      tol, maxit, ctypes.byref(iters), ctypes.byref(eta_dev)),
                          "solve")
        else:
            _native.check(lib.mf_factorize(h, None, None), "factorize")
            _native.check(lib.mf_solve_device(h, vp(X_dev.data_ptr()), args.nrhs, n, vp(perm_dev.data_ptr())),
                          "solve")

    def step_e2e():
        _native.check(lib.mf_assemble(h, ctypes.cast(nz_host.data_ptr(), pd)), "assemble")
        X_host.copy_(B_host)
        if mixed:
            _native.check(lib.mf_factorize_mixed(h, None, ctypes.byref(info), ctypes.byref(fp64)), "factorize")
            _native.check(lib.mf_solve_refined(h, ctypes.cast(X_host.data_ptr(), pd), args.nrhs, n, None, tol, maxit,
                                               ctypes.byref(iters), ctypes.byref(eta_dev)), "solve")
        else:
            _native.check(lib.mf_factorize(h, None, ctypes.byref(info)), "factorize")
            _native.check(lib.mf_solve(h, ctypes.cast(X_host.data_ptr(), pd), args.nrhs, n, None), "solve")

    with torch.cuda.stream(stream):
        step_device()
    stream.synchronize()
    X = X_dev.cpu().numpy().reshape(n, args.nrhs, order="F")
    eta = float(tm.backward_error(A, X, B).max())
    if profile_only:
        F.close()
        return {"profile_only": True, "mixed": mixed, "n": int(n), "backward_error": eta,
                "iterations": int(iters.value) if mixed else None}

    # perm for the host path is uploaded once (pattern constant)
    perm_np = np.ascontiguousarray(P.perm, dtype=np.int64)
    Xtmp = np.asfortranarray(B.copy())
    _native.check(lib.mf_solve(h, _native.ptrd(Xtmp), 0, n, _native.ptr64(perm_np)), "perm upload")
    if mixed:
        _native.check(lib.mf_solve_refined(h, _native.ptrd(Xtmp), 0, n, _native.ptr64(perm_np), tol, maxit,
                                           ctypes.byref(iters), ctypes.byref(eta_dev)), "perm upload")
    if info.value != 0 or not eta <= 1e-12:
        raise SystemExit(f"bench: check failed (mixed={mixed}, info={info.value}, backward error={eta})")

    # profiling pass (per-kernel events; not the timed pass)
    lib.mf_profile(h, 1)
    step_device()
    stream.synchronize()
    ms = (ctypes.c_double * NK)()
    ln = (ctypes.c_int64 * NK)()
    lib.mf_kernel_times(h, ms, ln)
    lib.mf_profile(h, 0)
    ktimes = {KERNEL_NAMES[i]: {"ms": ms[i], "launches": int(ln[i])} for i in range(NK)}
    launches_per_step = int(sum(ln[i] for i in range(NK)))
    enn, ena = exec_sizes(lib, h)
    fl = kernel_flops(enn, ena)

    # timed device-resident pass
    for _ in range(args.warmup):
        step_device()
    stream.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    clocks = Clocks(local)
    clocks.start()
    torch.cuda.synchronize()
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    evs[0].record(stream)
    its = []
    for i in range(args.steps):
        step_device()
        evs[i + 1].record(stream)
        its.append(int(iters.value))
    stream.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    step_ms = [evs[i].elapsed_time(evs[i + 1]) for i in range(args.steps)]
    total_s = sum(step_ms) / 1e3
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_s], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_s = float(t.item())
    value = world * args.steps / total_s
    Xt = X_dev.cpu().numpy().reshape(n, args.nrhs, order="F")
    eta_t = float(tm.backward_error(A, Xt, B).max())

    # e2e pass through the host-buffer C ABI
    for _ in range(args.warmup):
        step_e2e()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_ms = []
    for _ in range(args.steps):
        s0 = time.perf_counter()
        step_e2e()
        e2e_ms.append((time.perf_counter() - s0) * 1e3)
    e2e_total = time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([e2e_total], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total = float(t.item())
    e2e_value = world * args.steps / e2e_total
    Xe = X_host.numpy().reshape(n, args.nrhs, order="F")
    eta_e2e = float(tm.backward_error(A, Xe, B).max())
    F.close()
    del F
    torch.cuda.empty_cache()
    return {
        "value": value, "ms_per_step": 1e3 * total_s / args.steps,
        "p50_ms": float(np.percentile(step_ms, 50)), "p99_ms": float(np.percentile(step_ms, 99)),
        "backward_error": max(eta, eta_t), "iterations": its if mixed else None,
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(nz_host.numel() * 8 + n * args.nrhs * 8),
                "d2h_bytes_per_step": int(n * args.nrhs * 8 + 8), "backward_error": eta_e2e,
                "p50_ms": float(np.percentile(e2e_ms, 50)), "p99_ms": float(np.percentile(e2e_ms, 99))},
        "gpu_launches": launches_per_step * args.steps, "kernels": ktimes, "clocks": ck, "flops": fl,
    }


if __name__ == "__main__":
    main()
