"""Serving loop: factor + solve requests of mixed sizes and sparsity patterns
with continuous batching on one GPU.

The reference has no serving layer; it factors one matrix per call.  Here a
request is (pattern key, the matrix values on that pattern, right-hand
sides, arrival time).  The server

* caches the symbolic analysis of every pattern on the host (computed once)
  and, per pattern, batched device handles: a handle holds B copies of the
  pattern as one block-diagonal forest (``batch.block_symbolic``), so the B
  requests of a batch have their fronts merged at every tree level -- one
  grouped launch per level covers all of them -- and the factor and solve
  of the batch replay as CUDA graphs;
* admits requests into batches as they arrive and as handles free up:
  ``workers`` host threads each take the oldest waiting request's pattern,
  fill a batch with the waiting requests of that pattern (up to B) and run
  it on that handle's own CUDA stream, so batches of different patterns
  (and successive batches of one pattern) overlap on the device; the C ABI
  releases the GIL while it waits for the GPU;
* admits handles by device memory: a new handle is created only while the
  sum of the handles' device bytes stays under ``mem_cap`` (idle handles of
  other patterns are evicted, least recently used first); a handle larger
  than the cap on its own is admitted only when nothing else is resident;
* reports per-request latency (arrival to result on the host) and, in the
  mixed form, each request's normwise backward error (per-segment
  refinement: every request of a batch is refined until it alone meets the
  tolerance; the requests never share reductions).
"""
from __future__ import annotations

import collections
import ctypes
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import scipy.sparse as sp

from . import _native
from ._native import check, ptr64, ptrd
from .batch import block_symbolic
from .factorization import ChordalCholesky, ChordalLDLt
from .sparse import assembly_map
from .symbolic import symbolic


@dataclass
class Pattern:
    key: str
    A0: sp.csc_matrix          # a matrix with the pattern (any values)
    P: object
    S: object
    batch: int                 # requests per device handle
    ldlt: bool = False
    lo_src: np.ndarray = None  # one entry per stored lower-triangle value
    handles: list = field(default_factory=list)
    est_bytes: int = 0         # device bytes of one handle, once known
    creating: int = 0          # handles of this pattern being built outside the lock
    choice: tuple = None       # mixed form: per-level tcgen05/FFMA choice found by autotuning


@dataclass
class Request:
    rid: int
    key: str
    values: np.ndarray         # lower-triangle values in the pattern's CSC order
    B: np.ndarray              # n x k right-hand sides
    arrival: float = 0.0       # seconds after the stream start
    done: float = -1.0
    X: np.ndarray = None
    eta: float = -1.0
    batch_size: int = 0


@dataclass
class _Ticket:
    est: int  # bytes reserved for a handle being built


class _DeviceBatch:
    """One batched handle: B copies of a pattern as a forest, its own stream."""

    def __init__(self, pat: Pattern, mixed: bool, device: int, tol: float, maxit: int):
        import torch
        self.pat = pat
        B = pat.batch
        Pb, Sb, off = block_symbolic([(pat.P, pat.S)] * B)
        Ab = sp.block_diag([pat.A0] * B, format="csc")
        cls = ChordalLDLt if pat.ldlt else ChordalCholesky
        self.F = cls(Ab, Pb, Sb, device=device, nrhs_cap=16, mixed=mixed, tol=tol, maxit=maxit)
        self.offsets = off
        self.n1 = pat.S.n
        self.lib = _native.gpulib()
        self.h = self.F._handle.h
        check(self.lib.mf_set_segments(self.h, B, ptr64(np.ascontiguousarray(off))), "mf_set_segments")
        self.stream = torch.cuda.Stream(device=device)
        check(self.lib.mf_set_stream(self.h, ctypes.c_void_p(self.stream.cuda_stream)), "mf_set_stream")
        info = np.zeros(9, np.int64)
        self.lib.mf_info(self.h, info.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        self.bytes = int(info[6])
        self.mixed = mixed
        self.tol, self.maxit = tol, maxit
        self.perm = np.ascontiguousarray(Pb.perm, dtype=np.int64)
        if mixed and pat.choice is not None:
            self.F.set_kernel_choice(*pat.choice)
        self.busy = False
        self.last_used = 0.0
        self.nz = np.empty(pat.lo_src.size * B, np.float64)

    def run(self, reqs):
        """Factor and solve the requests (at most B) of one batch."""
        B = self.pat.batch
        m = self.pat.lo_src.size
        k = max(r.B.shape[1] for r in reqs)
        for i in range(B):
            src = reqs[i] if i < len(reqs) else reqs[-1]  # empty slots repeat the last request
            self.nz[i * m:(i + 1) * m] = src.values
        rhs = np.zeros((self.n1 * B, k), order="F")
        for i, r in enumerate(reqs):
            rhs[i * self.n1:(i + 1) * self.n1, :r.B.shape[1]] = r.B
        lib, h = self.lib, self.h
        check(lib.mf_assemble(h, ptrd(self.nz)), "mf_assemble")
        info = ctypes.c_int64(0)
        if self.mixed:
            fp64 = ctypes.c_int(0)
            check(lib.mf_factorize_mixed(h, None, ctypes.byref(info), ctypes.byref(fp64)), "mf_factorize_mixed")
        else:
            check(lib.mf_factorize(h, None, ctypes.byref(info)), "mf_factorize")
        if info.value != 0:
            raise RuntimeError(f"factorization failed at column {info.value}")
        if self.mixed:
            it = ctypes.c_int(0)
            eta = ctypes.c_double(0.0)
            check(lib.mf_solve_refined(h, ptrd(rhs), k, rhs.shape[0], ptr64(self.perm), self.tol, self.maxit,
                                       ctypes.byref(it), ctypes.byref(eta)), "mf_solve_refined")
            seg = np.zeros(B, np.float64)
            check(lib.mf_segment_errors(h, ptrd(seg)), "mf_segment_errors")
        else:
            check(lib.mf_solve(h, ptrd(rhs), k, rhs.shape[0], ptr64(self.perm)), "mf_solve")
            seg = None
        for i, r in enumerate(reqs):
            r.X = rhs[i * self.n1:(i + 1) * self.n1, :r.B.shape[1]].copy()
            r.eta = float(seg[i]) if seg is not None else -1.0
            r.batch_size = len(reqs)

    def close(self):
        self.F.close()


class Server:
    def __init__(self, *, mixed=True, device=0, mem_cap=120e9, workers=4, tol=1e-12, maxit=100, autotune=True):
        self.mixed = mixed
        self.autotune = autotune
        self.device = device
        self.mem_cap = mem_cap
        self.workers = workers
        self.tol, self.maxit = tol, maxit
        self.patterns: dict[str, Pattern] = {}
        self.lock = threading.Lock()
        self.cv = threading.Condition(self.lock)
        self.bytes = 0
        self.reserved = 0  # bytes of handles being built

    # -- patterns ----------------------------------------------------------
    def add_pattern(self, key, A0, order="amf", batch=1, ldlt=False, symbolic_result=None):
        """Symbolic analysis of a pattern, once (cached by key); an analysis
        already at hand is passed as ``symbolic_result=(P, S)``."""
        if key in self.patterns:
            return self.patterns[key]
        A0 = sp.csc_matrix(A0)
        P, S = symbolic_result if symbolic_result is not None else symbolic(A0, alg=order)
        Lo, _ = assembly_map(S, P.invp, A0)
        pat = Pattern(key, A0, P, S, batch, ldlt, np.arange(Lo.nnz))
        self.patterns[key] = pat
        return pat

    def lower_values(self, key, A):
        """The stored lower-triangle values of A (pattern `key`) in the order the
        device assembly expects."""
        L = sp.tril(sp.csc_matrix(A), format="csc")
        L.sort_indices()
        return np.ascontiguousarray(L.data, dtype=np.float64)

    # -- device handles ----------------------------------------------------
    def _acquire(self, pat: Pattern):
        """With the lock held: a free handle of `pat` (marked busy); or, when a
        new handle may be built under the memory cap, a _Ticket that reserves
        its slot and bytes (the caller builds it with _create, outside the
        lock, so that building -- seconds for a large pattern -- never stalls
        the other workers); or None if neither is possible now."""
        for hd in pat.handles:
            if not hd.busy:
                hd.busy = True
                return hd
        if len(pat.handles) + pat.creating >= 2:  # two per pattern: one runs while the next batch fills
            return None
        # evict idle handles of other patterns while over the cap (least recently used first)
        est = max([hd.bytes for hd in pat.handles] + [pat.est_bytes])
        if not self._make_room(pat, est):
            return None
        pat.creating += 1
        self.reserved += est
        return _Ticket(est)

    def _make_room(self, pat, need):
        """With the lock held: evict idle handles of other patterns until `need`
        more bytes fit under the cap (or nothing else is resident)."""
        while self.bytes + self.reserved + need > self.mem_cap and self.bytes + self.reserved > 0:
            idle = [(hd.last_used, p, hd) for p in self.patterns.values() for hd in p.handles
                    if not hd.busy and p is not pat]
            if not idle:
                return False
            _, p, hd = min(idle, key=lambda x: x[0])
            p.handles.remove(hd)
            self.bytes -= hd.bytes
            hd.close()
        return True

    def _create(self, pat: Pattern, ticket):
        """Without the lock: build the handle a ticket reserved and admit it
        (marked busy); None if the cap turns it away once its true size is
        known (the caller retries later)."""
        try:
            hd = _DeviceBatch(pat, self.mixed, self.device, self.tol, self.maxit)
        except BaseException:
            with self.cv:
                pat.creating -= 1
                self.reserved -= ticket.est
                self.cv.notify_all()
            raise
        with self.cv:
            pat.creating -= 1
            self.reserved -= ticket.est
            pat.est_bytes = hd.bytes
            if not self._make_room(pat, hd.bytes):
                self.cv.notify_all()
                admit = False
            else:
                hd.busy = True
                pat.handles.append(hd)
                self.bytes += hd.bytes
                self.cv.notify_all()
                admit = True
        if not admit:
            hd.close()  # the next attempt evicts idle handles first
            return None
        return hd

    def _get(self, pat: Pattern):
        """A handle of `pat` for single-threaded use (warm-up): free or built now."""
        with self.cv:
            got = self._acquire(pat)
        if isinstance(got, _Ticket):
            return self._create(pat, got)
        return got

    def warm(self, keys=None, per_pattern=1):
        """Create up to ``per_pattern`` handles per pattern (at most 2) and run
        a throw-away batch through each, so graphs and tensor maps exist
        before timing; in the mixed form the pattern's per-level kernel
        choice is autotuned on its first handle and every later handle of
        the pattern starts with it."""
        for key in keys or list(self.patterns):
            pat = self.patterns[key]
            got = []
            for _ in range(max(1, min(2, per_pattern))):
                hd = self._get(pat)
                if hd is None:
                    break
                got.append(hd)
                A = pat.A0
                r = Request(-1, key, self.lower_values(key, A), np.ones((pat.S.n, 1)))
                hd.run([r])
                if self.mixed and self.autotune and pat.choice is None:
                    t = hd.F.autotune(2)
                    pat.choice = (t["tc_steps"], t["tc_syrk"])
                    for other in pat.handles:
                        if other is not hd:
                            other.F.set_kernel_choice(*pat.choice)
                    hd.run([r])
            for hd in got:
                hd.busy = False

    # -- the loop ----------------------------------------------------------
    def serve(self, requests, realtime=True, timeout=600.0):
        """Run a stream of requests (sorted by arrival); returns them with
        completion times and solutions filled in.  Raises TimeoutError if the
        stream is not done after `timeout` seconds (batches already on the
        GPU finish first)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: dict[str, collections.deque] = {k: collections.deque() for k in self.patterns}
        total = len(pending)
        finished = []
        t0 = time.perf_counter()
        errors = []

        def now():
            return time.perf_counter() - t0

        def admit_arrivals():
            t = now()
            while pending and (not realtime or pending[0].arrival <= t):
                r = pending.popleft()
                waiting[r.key].append(r)

        def worker():
            while True:
                with self.cv:
                    while True:
                        if len(finished) + sum(len(q) for q in waiting.values()) == total and not any(
                                waiting.values()) and not pending:
                            return
                        if errors:
                            return
                        admit_arrivals()
                        # oldest waiting request first; its pattern's batch takes the others waiting
                        cands = sorted((q[0].arrival, k) for k, q in waiting.items() if q)
                        job = None
                        for _, k in cands:
                            got = self._acquire(self.patterns[k])
                            if got is not None:
                                q = waiting[k]
                                batch = [q.popleft() for _ in range(min(len(q), self.patterns[k].batch))]
                                job = (got, k, batch)
                                break
                        if job is not None:
                            break
                        if not pending and not any(waiting.values()):
                            return
                        timeout = 0.0005
                        if pending and not any(waiting.values()) and realtime:
                            timeout = max(0.0, min(0.01, pending[0].arrival - now()))
                        self.cv.wait(timeout)
                got, k, batch = job
                try:
                    hd = self._create(self.patterns[k], got) if isinstance(got, _Ticket) else got
                except Exception as e:  # noqa: BLE001
                    with self.cv:
                        errors.append(e)
                        self.cv.notify_all()
                    return
                if hd is None:  # turned away by the cap: back to the front of the queue
                    with self.cv:
                        waiting[k].extendleft(reversed(batch))
                        self.cv.notify_all()
                    continue
                try:
                    hd.run(batch)
                except Exception as e:  # noqa: BLE001
                    with self.cv:
                        errors.append(e)
                        self.cv.notify_all()
                    return
                t = now()
                with self.cv:
                    for r in batch:
                        r.done = t
                        finished.append(r)
                    hd.busy = False
                    hd.last_used = t
                    self.cv.notify_all()

        threads = [threading.Thread(target=worker, daemon=True) for _ in range(self.workers)]
        for th in threads:
            th.start()
        deadline = time.perf_counter() + timeout
        for th in threads:
            th.join(max(0.0, deadline - time.perf_counter()))
        if any(th.is_alive() for th in threads):
            with self.cv:
                errors.append(TimeoutError(f"serve: {total - len(finished)} of {total} requests not done "
                                           f"after {timeout:.0f} s"))
                self.cv.notify_all()
            for th in threads:
                th.join()
        if errors:
            raise errors[0]
        self.wall = now()
        return finished

    def close(self):
        for p in self.patterns.values():
            for hd in p.handles:
                hd.close()
            p.handles.clear()
        self.bytes = 0


def latency_stats(done):
    lat = np.array([r.done - r.arrival for r in done]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}
