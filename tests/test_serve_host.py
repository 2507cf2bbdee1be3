"""Host logic of the serving loop, with the device batch replaced by a fake
(no GPU): every request completes once, requests of one pattern share
batches, the memory cap evicts idle handles, and a handle larger than the
cap runs alone instead of waiting forever."""
import time

import numpy as np

import multifrontal as mf
from multifrontal import serve
from multifrontal import testmatrices as tm


class FakeBatch:
    def __init__(self, pat, mixed, device, tol, maxit):
        self.pat = pat
        self.bytes = pat.S.n * 1000 * pat.batch
        self.busy = False
        self.last_used = 0.0

    def run(self, reqs):
        time.sleep(0.001)
        for r in reqs:
            r.X = np.zeros_like(r.B)
            r.eta = 0.0
            r.batch_size = len(reqs)

    def close(self):
        pass


PATS = {
    "g2d12": (lambda s: tm.grid_laplacian(12, 12, seed=s), "amf", 4),
    "g2d20": (lambda s: tm.grid_laplacian(20, 20, seed=s), "amf", 4),
    "g3d6": (lambda s: tm.grid_laplacian(6, 6, 6, seed=s), "natural", 2),
}


def _server(monkeypatch, workers):
    monkeypatch.setattr(serve, "_DeviceBatch", FakeBatch)
    srv = serve.Server(mixed=False, workers=workers)
    for k, (gen, order, batch) in PATS.items():
        srv.add_pattern(k, gen(0), order=order, batch=batch)
    return srv


def _requests(srv, count, seed, spacing=0.0):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        k = list(PATS)[rng.integers(len(PATS))]
        A = PATS[k][0](1000 + i)
        reqs.append(serve.Request(i, k, srv.lower_values(k, A), np.ones((A.shape[0], 2)), arrival=spacing * i))
    return reqs


def test_all_requests_complete_and_batch(monkeypatch):
    srv = _server(monkeypatch, workers=3)
    done = srv.serve(_requests(srv, 40, seed=1), realtime=False, timeout=30)
    assert sorted(r.rid for r in done) == list(range(40))
    assert max(r.batch_size for r in done) > 1
    for r in done:
        assert r.batch_size <= srv.patterns[r.key].batch
    st = serve.latency_stats(done)
    assert st["p99_ms"] >= st["p50_ms"] >= 0


def test_memory_cap_evicts_and_oversize_runs_alone(monkeypatch):
    srv = _server(monkeypatch, workers=1)
    srv.warm(["g2d12"])
    srv.mem_cap = srv.bytes * 1.5  # g2d20's handle alone exceeds the cap
    done = srv.serve(_requests(srv, 15, seed=3), realtime=False, timeout=30)
    assert len(done) == 15
    resident = [h for p in srv.patterns.values() for h in p.handles]
    assert len(resident) == 1 or srv.bytes <= srv.mem_cap


def test_realtime_arrivals_are_respected(monkeypatch):
    srv = _server(monkeypatch, workers=2)
    done = srv.serve(_requests(srv, 10, seed=5, spacing=0.01), realtime=True, timeout=30)
    assert all(r.done >= r.arrival for r in done)


class FakeFactor:
    """Stands in for a mixed factorization: records the kernel choice it is given."""

    def __init__(self):
        self.choice = None
        self.tuned = 0

    def autotune(self, reps):
        self.tuned += 1
        return {"tc_steps": np.array([1, 0, 1], np.int32), "tc_syrk": np.array([1, 1, 0], np.int32)}

    def set_kernel_choice(self, tc_steps, tc_syrk):
        self.choice = (np.asarray(tc_steps).copy(), np.asarray(tc_syrk).copy())


class FakeMixedBatch(FakeBatch):
    def __init__(self, pat, mixed, device, tol, maxit):
        super().__init__(pat, mixed, device, tol, maxit)
        self.F = FakeFactor()
        if mixed and pat.choice is not None:
            self.F.set_kernel_choice(*pat.choice)


def test_warm_autotunes_once_and_shares_the_choice(monkeypatch):
    """Mixed serving: warming two handles of a pattern autotunes the first
    one only; the pattern keeps the choice and the second handle gets it."""
    monkeypatch.setattr(serve, "_DeviceBatch", FakeMixedBatch)
    srv = serve.Server(mixed=True, workers=2)
    gen, order, batch = PATS["g2d12"]
    srv.add_pattern("g2d12", gen(0), order=order, batch=batch)
    srv.warm(["g2d12"], per_pattern=2)
    pat = srv.patterns["g2d12"]
    assert len(pat.handles) == 2 and not any(h.busy for h in pat.handles)
    assert sum(h.F.tuned for h in pat.handles) == 1
    assert pat.choice is not None
    tuned = [h for h in pat.handles if h.F.tuned][0]
    other = [h for h in pat.handles if h is not tuned][0]
    np.testing.assert_array_equal(other.F.choice[0], pat.choice[0])
    np.testing.assert_array_equal(other.F.choice[1], pat.choice[1])


def test_add_pattern_accepts_a_symbolic_result(monkeypatch):
    monkeypatch.setattr(serve, "_DeviceBatch", FakeBatch)
    srv = serve.Server(mixed=False, workers=1)
    A = tm.grid_laplacian(10, 10, seed=1)
    P, S = mf.symbolic(A, alg="amf")
    pat = srv.add_pattern("p", A, symbolic_result=(P, S))
    assert pat.S is S and pat.P is P


class SlowBuildBatch(FakeBatch):
    """Building a handle of pattern g3d6 takes half a second."""

    def __init__(self, pat, mixed, device, tol, maxit):
        if pat.key == "g3d6":
            time.sleep(0.5)
        super().__init__(pat, mixed, device, tol, maxit)


def test_building_a_handle_does_not_stall_other_patterns(monkeypatch):
    """A new handle is built outside the scheduler lock: while one worker
    builds the slow pattern's handle, the other worker keeps serving the
    pattern whose handle already exists."""
    monkeypatch.setattr(serve, "_DeviceBatch", SlowBuildBatch)
    srv = serve.Server(mixed=False, workers=2)
    for k, (gen, order, batch) in PATS.items():
        srv.add_pattern(k, gen(0), order=order, batch=batch)
    srv.warm(["g2d12"])
    A3 = PATS["g3d6"][0](5)
    reqs = [serve.Request(0, "g3d6", srv.lower_values("g3d6", A3), np.ones((A3.shape[0], 1)), arrival=0.0)]
    for i in range(1, 13):
        A = PATS["g2d12"][0](100 + i)
        reqs.append(serve.Request(i, "g2d12", srv.lower_values("g2d12", A), np.ones((A.shape[0], 1)),
                                  arrival=1e-6 * i))
    done = srv.serve(reqs, realtime=False, timeout=30)
    assert len(done) == 13
    slow = [r for r in done if r.key == "g3d6"][0]
    fast_done = max(r.done for r in done if r.key == "g2d12")
    assert fast_done < slow.done - 0.2, (fast_done, slow.done)
    assert srv.reserved == 0 and all(p.creating == 0 for p in srv.patterns.values())


def test_cap_turns_a_new_handle_away_and_the_batch_is_served_later(monkeypatch):
    """A handle whose true size does not fit is closed and its requests go back
    to the queue; they are served once the cap allows."""
    monkeypatch.setattr(serve, "_DeviceBatch", FakeBatch)
    srv = _server(monkeypatch, workers=2)
    srv.warm(["g2d12"])
    srv.mem_cap = srv.bytes * 1.2
    done = srv.serve(_requests(srv, 20, seed=9), realtime=False, timeout=30)
    assert sorted(r.rid for r in done) == list(range(20))
    assert srv.reserved == 0 and all(p.creating == 0 for p in srv.patterns.values())
