"""Serving loop: factor + solve requests of mixed sizes and sparsity patterns
with continuous batching on one GPU.

The reference has no serving layer; it factors one matrix per call.  Here a
request is (pattern key, the matrix values on that pattern, right-hand
sides, arrival time).  The server

* caches the symbolic analysis of every pattern on the host (computed once);
* forms admission rounds: the oldest waiting request opens a round, which
  takes the other waiting requests in arrival order -- of any pattern of the
  same size class -- up to each pattern's per-round limit and the round's
  memory budget.  The round's requests are factored and solved as ONE
  forest (their ChordalSymbolic arrays concatenated, ``batch.block_symbolic``):
  the fronts of all of them, whatever their patterns, are merged at every
  tree level into one grouped launch, and the factorization and the solve
  replay as CUDA graphs.  The forest's composition (count per pattern, each
  count rounded down to a power of two so that few distinct compositions
  occur; the requests left over wait for the next round) keys a cache of
  device handles, so a composition is planned and allocated once;
* admits each request by its own memory: the front-stack + factor bytes of
  its pattern (``request_bytes``: the factor, the LIFO update-matrix stack
  bound and the largest frontal matrix of ChordalSymbolic,
  src/Multifrontal.jl/src/chordal_symbolic.jl:354-367); a round's requests
  must fit the round budget, and a new handle is built only while the
  resident handles plus its estimated size stay under ``mem_cap`` (idle
  handles are evicted, least recently used first; a handle larger than the
  cap on its own runs only when nothing else is resident);
* runs rounds on ``workers`` host threads, each handle on its own CUDA
  stream, so rounds overlap on the device; the C ABI releases the GIL while
  it waits for the GPU.  Requests that arrive while others are on the GPU
  open or join the next round as soon as a handle is free (continuous
  batching); a round never repeats a request to fill a slot;
* reports per-request latency (arrival to result on the host) and, in the
  mixed form, each request's normwise backward error (per-segment
  refinement: every request of a round is refined until it alone meets the
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
    batch: int                 # most requests of this pattern in one round
    ldlt: bool = False
    nnz_lower: int = 0         # stored lower-triangle values per request
    size_class: int = 0        # rounds merge patterns of one class
    req_bytes: int = 0         # admission bytes of one request (request_bytes)


@dataclass
class Request:
    rid: int
    key: str
    values: np.ndarray         # lower-triangle values in the pattern's CSC order (or None: see make_values)
    B: np.ndarray              # n x k right-hand sides
    arrival: float = 0.0       # seconds after the stream start
    done: float = -1.0
    X: np.ndarray = None
    eta: float = -1.0
    batch_size: int = 0        # requests in its round
    make_values: object = None  # callable producing `values` when the request is admitted (fresh coefficients)
    make_rhs: object = None    # callable producing `B` when the request is admitted
    keep: bool = True          # keep X (and B) after serving; False drops them once the request is done
    coef_seed: int = None      # caller's bookkeeping (the seed its coefficients came from)


def request_bytes(S, nnz_lower, mixed):
    """Device bytes one request of a pattern is admitted by: its factor
    (sum nn^2 + nn na values), the LIFO update-matrix stack bound nMval and
    the largest frontal matrix nFval^2 of its ChordalSymbolic
    (chordal_symbolic.jl:354-367), in the factor's precision, plus its
    values and the refinement vectors."""
    w = 4 if mixed else 8
    return int(w * (S.ndz + S.nlz + S.nMval + S.nFval * S.nFval) + 8 * (nnz_lower + 8 * S.n * 16))


def _pow2_floor(c):
    p = 1
    while p * 2 <= c:
        p *= 2
    return p


class _DeviceBatch:
    """One device handle for a composition: the requests of a round, of one
    or several patterns, as one forest on the handle's own stream."""

    def __init__(self, comp, patterns, mixed: bool, device: int, tol: float, maxit: int):
        self.comp = comp
        members = [patterns[k] for k, c in comp for _ in range(c)]
        self.members = members
        Pb, Sb, off = block_symbolic([(p.P, p.S) for p in members])
        Ab = sp.block_diag([p.A0 for p in members], format="csc")
        ldlt = members[0].ldlt
        cls = ChordalLDLt if ldlt else ChordalCholesky
        self.F = cls(Ab, Pb, Sb, device=device, nrhs_cap=16, mixed=mixed, tol=tol, maxit=maxit)
        self.offsets = off
        self.lib = _native.gpulib()
        self.h = self.F._handle.h
        check(self.lib.mf_set_segments(self.h, len(members), ptr64(np.ascontiguousarray(off))), "mf_set_segments")
        # the handle keeps the non-blocking stream the library created for it:
        # torch.cuda.Stream() hands out streams from a fixed per-device pool,
        # so past its size two handles would share a stream and two workers
        # could capture graphs on it at once
        info = np.zeros(9, np.int64)
        self.lib.mf_info(self.h, info.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        self.bytes = int(info[6])
        self.mixed = mixed
        self.tol, self.maxit = tol, maxit
        self.perm = np.ascontiguousarray(Pb.perm, dtype=np.int64)
        self.busy = False
        self.last_used = 0.0
        self.nzoff = np.concatenate([[0], np.cumsum([p.nnz_lower for p in members])]).astype(np.int64)
        self.nz = np.empty(int(self.nzoff[-1]), np.float64)

    def run(self, reqs):
        """Factor and solve the requests of one round, in composition order
        (pattern by pattern, arrival order inside a pattern)."""
        assert len(reqs) == len(self.members)
        k = max(r.B.shape[1] for r in reqs)
        n = self.F.S.n
        rhs = np.zeros((n, k), order="F")
        for i, r in enumerate(reqs):
            assert r.key == self.members[i].key
            self.nz[self.nzoff[i]:self.nzoff[i + 1]] = r.values
            rhs[self.offsets[i]:self.offsets[i + 1], :r.B.shape[1]] = r.B
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
            check(lib.mf_solve_refined(h, ptrd(rhs), k, n, ptr64(self.perm), self.tol, self.maxit,
                                       ctypes.byref(it), ctypes.byref(eta)), "mf_solve_refined")
            seg = np.zeros(len(reqs), np.float64)
            check(lib.mf_segment_errors(h, ptrd(seg)), "mf_segment_errors")
        else:
            check(lib.mf_solve(h, ptrd(rhs), k, n, ptr64(self.perm)), "mf_solve")
            seg = None
        for i, r in enumerate(reqs):
            r.X = rhs[self.offsets[i]:self.offsets[i + 1], :r.B.shape[1]].copy()
            r.eta = float(seg[i]) if seg is not None else -1.0
            r.batch_size = len(reqs)

    def close(self):
        self.F.close()


@dataclass
class _Ticket:
    comp: tuple
    est: int  # bytes reserved for a handle being built


class Server:
    def __init__(self, *, mixed=True, device=0, mem_cap=120e9, workers=4, tol=1e-12, maxit=100,
                 round_budget=None, max_members=32):
        self.mixed = mixed
        self.device = device
        self.mem_cap = mem_cap
        self.workers = workers
        self.tol, self.maxit = tol, maxit
        self.round_budget = round_budget if round_budget is not None else mem_cap / 4
        self.max_members = max_members
        self.patterns: dict[str, Pattern] = {}
        self.handles: dict[tuple, list] = {}   # composition -> resident handles
        self.creating: dict[tuple, int] = {}   # composition -> handles being built
        self.est: dict[tuple, int] = {}        # composition -> device bytes of its handle, once known
        self.lock = threading.Lock()
        self.cv = threading.Condition(self.lock)
        self.bytes = 0
        self.reserved = 0  # bytes of handles being built
        self.rounds = []   # compositions of the rounds run by the last serve()

    # -- patterns ----------------------------------------------------------
    def add_pattern(self, key, A0, order="amf", batch=1, ldlt=False, symbolic_result=None, size_class=None):
        """Symbolic analysis of a pattern, once (cached by key); an analysis
        already at hand is passed as ``symbolic_result=(P, S)``.  ``batch``:
        most requests of this pattern in one round; ``size_class``: rounds
        merge patterns of one class (default: by factor size, decades of
        stored factor entries)."""
        if key in self.patterns:
            return self.patterns[key]
        A0 = sp.csc_matrix(A0)
        P, S = symbolic_result if symbolic_result is not None else symbolic(A0, alg=order)
        Lo, _ = assembly_map(S, P.invp, A0)
        if size_class is None:
            size_class = int(np.log10(max(S.ndz + S.nlz, 1)))
        pat = Pattern(key, A0, P, S, batch, ldlt, int(Lo.nnz), size_class,
                      request_bytes(S, int(Lo.nnz), self.mixed))
        self.patterns[key] = pat
        return pat

    def lower_values(self, key, A):
        """The stored lower-triangle values of A (pattern `key`) in the order the
        device assembly expects."""
        L = sp.tril(sp.csc_matrix(A), format="csc")
        L.sort_indices()
        return np.ascontiguousarray(L.data, dtype=np.float64)

    def estimate_bytes(self, comp):
        """Device bytes a handle for `comp` would take, estimated on the host
        from the requests' admission bytes and the plan of its forest."""
        if comp in self.est:
            return self.est[comp]
        return int(1.5 * sum(self.patterns[k].req_bytes * c for k, c in comp))

    # -- rounds and handles --------------------------------------------------
    def _form_round(self, waiting):
        """With the lock held: the composition and requests of the next round,
        opened by the oldest waiting request (None if nothing waits)."""
        heads = [(q[0].arrival, k) for k, q in waiting.items() if q]
        if not heads:
            return None
        _, k0 = min(heads)
        cls = (self.patterns[k0].size_class, self.patterns[k0].ldlt)
        # waiting requests of the class in arrival order, within the limits
        cand = sorted((r.arrival, r.rid, k) for k, q in waiting.items()
                      if (self.patterns[k].size_class, self.patterns[k].ldlt) == cls for r in q)
        take = collections.Counter()
        budget = self.round_budget
        used = 0
        members = 0
        for _, _, k in cand:
            p = self.patterns[k]
            if take[k] >= p.batch or members >= self.max_members:
                continue
            if members > 0 and used + p.req_bytes > budget:
                continue
            take[k] += 1
            used += p.req_bytes
            members += 1
        comp = tuple(sorted((k, _pow2_floor(c)) for k, c in take.items()))
        return comp

    def _acquire(self, comp):
        """With the lock held: a free handle of `comp` (marked busy); or, when a
        new one may be built under the memory cap, a _Ticket reserving its
        bytes (built with _create outside the lock); or None."""
        for hd in self.handles.get(comp, []):
            if not hd.busy:
                hd.busy = True
                return hd
        if len(self.handles.get(comp, [])) + self.creating.get(comp, 0) >= self.workers:
            return None
        est = self.estimate_bytes(comp)
        if not self._make_room(comp, est):
            return None
        self.creating[comp] = self.creating.get(comp, 0) + 1
        self.reserved += est
        return _Ticket(comp, est)

    def _make_room(self, comp, need):
        """With the lock held: evict idle handles of other compositions until
        `need` more bytes fit under the cap (or nothing else is resident)."""
        while self.bytes + self.reserved + need > self.mem_cap and self.bytes + self.reserved > 0:
            idle = [(hd.last_used, c, hd) for c, hs in self.handles.items() for hd in hs
                    if not hd.busy and c != comp]
            if not idle:
                return False
            _, c, hd = min(idle, key=lambda x: x[0])
            self.handles[c].remove(hd)
            self.bytes -= hd.bytes
            hd.close()
        return True

    def _create(self, ticket):
        """Without the lock: build the handle a ticket reserved and admit it
        (marked busy); None if the cap turns it away once its true size is
        known (the caller retries later)."""
        comp = ticket.comp
        try:
            hd = _DeviceBatch(comp, self.patterns, self.mixed, self.device, self.tol, self.maxit)
        except BaseException:
            with self.cv:
                self.creating[comp] -= 1
                self.reserved -= ticket.est
                self.cv.notify_all()
            raise
        with self.cv:
            self.creating[comp] -= 1
            self.reserved -= ticket.est
            self.est[comp] = hd.bytes
            if not self._make_room(comp, hd.bytes):
                self.cv.notify_all()
                admit = False
            else:
                hd.busy = True
                self.handles.setdefault(comp, []).append(hd)
                self.bytes += hd.bytes
                self.cv.notify_all()
                admit = True
        if not admit:
            hd.close()
            return None
        return hd

    def _get(self, comp):
        with self.cv:
            got = self._acquire(comp)
        if isinstance(got, _Ticket):
            return self._create(got)
        return got

    def warm(self, keys=None, per_pattern=1, counts=None):
        """Build handles for single-pattern compositions (count 1 and, for a
        pattern whose rounds can hold more, its largest power of two) and run
        a throw-away round through each, so plans, graphs and tensor maps
        exist before timing.  ``per_pattern`` handles per composition (at
        most one per worker, the most the loop keeps)."""
        for key in keys or list(self.patterns):
            pat = self.patterns[key]
            cs = counts or sorted({1, _pow2_floor(pat.batch)})
            for c in cs:
                comp = ((key, c),)
                got = []
                for _ in range(max(1, min(self.workers, per_pattern))):
                    hd = self._get(comp)
                    if hd is None:
                        break
                    got.append(hd)
                    reqs = [Request(-1, key, self.lower_values(key, pat.A0), np.ones((pat.S.n, 1)))
                            for _ in range(c)]
                    hd.run(reqs)
                for hd in got:
                    hd.busy = False

    # -- the loop ----------------------------------------------------------
    def serve(self, requests, realtime=True, timeout=600.0):
        """Run a stream of requests (sorted by arrival); returns them with
        completion times and solutions filled in.  Raises TimeoutError if the
        stream is not done after `timeout` seconds (rounds already on the
        GPU finish first)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        waiting: dict[str, collections.deque] = {k: collections.deque() for k in self.patterns}
        total = len(pending)
        finished = []
        self.rounds = []
        t0 = time.perf_counter()
        errors = []

        def now():
            return time.perf_counter() - t0

        def admit_arrivals():
            t = now()
            while pending and (not realtime or pending[0].arrival <= t):
                r = pending.popleft()
                waiting[r.key].append(r)

        def take(comp):
            return [waiting[k].popleft() for k, c in comp for _ in range(c)]

        def worker():
            while True:
                with self.cv:
                    while True:
                        if errors:
                            return
                        admit_arrivals()
                        if not pending and not any(waiting.values()):
                            return
                        job = None
                        comp = self._form_round(waiting)
                        if comp is not None:
                            got = self._acquire(comp)
                            exists = len(self.handles.get(comp, [])) + self.creating.get(comp, 0) > 0
                            if got is None and not exists and (len(comp) > 1 or comp[0][1] > 1):
                                # the composition has no handle and none can be built
                                # under the cap now: the oldest request's pattern alone
                                # (while its handles are only busy, the round waits for one)
                                heads = [(q[0].arrival, k) for k, q in waiting.items() if q]
                                k0 = min(heads)[1]
                                comp = ((k0, 1),)
                                got = self._acquire(comp)
                            if got is not None:
                                job = (got, comp, take(comp))
                        if job is not None:
                            break
                        timeout = 0.0005
                        if pending and not any(waiting.values()) and realtime:
                            timeout = max(0.0, min(0.01, pending[0].arrival - now()))
                        self.cv.wait(timeout)
                got, comp, batch = job
                try:
                    for r in batch:  # fresh coefficients are generated when the request is admitted
                        if r.values is None and r.make_values is not None:
                            r.values = r.make_values()
                        if r.B is None and r.make_rhs is not None:
                            r.B = r.make_rhs()
                    hd = self._create(got) if isinstance(got, _Ticket) else got
                except Exception as e:  # noqa: BLE001
                    with self.cv:
                        errors.append(e)
                        self.cv.notify_all()
                    return
                if hd is None:  # turned away by the cap: back to the front of the queues
                    with self.cv:
                        for r in reversed(batch):
                            waiting[r.key].appendleft(r)
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
                        if r.make_values is not None:
                            r.values = None  # fresh values are not kept after the request is served
                        if not r.keep:
                            r.X = None
                            if r.make_rhs is not None:
                                r.B = None
                        finished.append(r)
                    self.rounds.append(comp)
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
        for hs in self.handles.values():
            for hd in hs:
                hd.close()
        self.handles.clear()
        self.bytes = 0


def latency_stats(done):
    lat = np.array([r.done - r.arrival for r in done]) * 1e3
    return {"p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean())}
