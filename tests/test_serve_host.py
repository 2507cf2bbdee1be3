"""Host logic of the serving loop, with the device handle replaced by a fake
(no GPU): every request completes once, rounds merge requests of different
patterns of one size class, counts per pattern are powers of two within the
pattern's limit, no request is repeated to fill a round, the memory cap
evicts idle handles and is respected before a handle is built, and a handle
larger than the cap runs alone instead of waiting forever."""
import time

import numpy as np

from multifrontal import serve
from multifrontal import testmatrices as tm


class FakeBatch:
    built = []

    def __init__(self, comp, patterns, mixed, device, tol, maxit):
        self.comp = comp
        self.members = [patterns[k] for k, c in comp for _ in range(c)]
        self.bytes = sum(p.S.n * 1000 for p in self.members)
        self.busy = False
        self.last_used = 0.0
        FakeBatch.built.append(self)

    def run(self, reqs):
        assert len(reqs) == len(self.members)
        assert [r.key for r in reqs] == [p.key for p in self.members]
        assert len({id(r) for r in reqs}) == len(reqs)  # never the same request twice
        time.sleep(0.001)
        for r in reqs:
            r.X = np.zeros_like(r.B)
            r.eta = 0.0
            r.batch_size = len(reqs)

    def close(self):
        pass


PATS = {
    "g2d12": (lambda s: tm.grid_laplacian(12, 12, seed=s), "amf", 4),
    "g2d14": (lambda s: tm.grid_laplacian(14, 14, seed=s), "amf", 4),
    "g3d6": (lambda s: tm.grid_laplacian(6, 6, 6, seed=s), "natural", 2),
}


def _server(monkeypatch, workers, **kw):
    monkeypatch.setattr(serve, "_DeviceBatch", FakeBatch)
    srv = serve.Server(mixed=False, workers=workers, **kw)
    for k, (gen, order, batch) in PATS.items():
        srv.add_pattern(k, gen(0), order=order, batch=batch, size_class=0)
    return srv


def _requests(srv, count, seed, spacing=0.0):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        k = list(PATS)[rng.integers(len(PATS))]
        A = PATS[k][0](1000 + i)
        reqs.append(serve.Request(i, k, srv.lower_values(k, A), np.ones((A.shape[0], 2)), arrival=spacing * i))
    return reqs


def test_all_requests_complete_in_merged_rounds(monkeypatch):
    srv = _server(monkeypatch, workers=3)
    done = srv.serve(_requests(srv, 60, seed=1), realtime=False, timeout=30)
    assert sorted(r.rid for r in done) == list(range(60))
    assert max(r.batch_size for r in done) > 1
    # some round merged requests of different patterns into one forest
    assert any(len(c) > 1 for c in srv.rounds)
    for comp in srv.rounds:
        for k, c in comp:
            assert c <= srv.patterns[k].batch and (c & (c - 1)) == 0  # within the limit, a power of two
    st = serve.latency_stats(done)
    assert st["p99_ms"] >= st["p50_ms"] >= 0


def test_size_classes_are_not_merged(monkeypatch):
    srv = _server(monkeypatch, workers=2)
    srv.patterns["g3d6"].size_class = 1
    srv.serve(_requests(srv, 40, seed=2), realtime=False, timeout=30)
    for comp in srv.rounds:
        keys = {k for k, _ in comp}
        assert not ("g3d6" in keys and len(keys) > 1)


def test_round_budget_limits_admitted_bytes(monkeypatch):
    srv = _server(monkeypatch, workers=1)
    one = max(p.req_bytes for p in srv.patterns.values())
    srv.round_budget = 2.5 * one
    srv.serve(_requests(srv, 30, seed=4), realtime=False, timeout=30)
    for comp in srv.rounds:
        used = sum(srv.patterns[k].req_bytes * c for k, c in comp)
        assert used <= srv.round_budget or sum(c for _, c in comp) == 1


def test_memory_cap_evicts_and_oversize_runs_alone(monkeypatch):
    srv = _server(monkeypatch, workers=1)
    srv.warm(["g2d12"], counts=[1])
    srv.mem_cap = srv.bytes * 1.5
    done = srv.serve(_requests(srv, 15, seed=3), realtime=False, timeout=30)
    assert len(done) == 15
    assert srv.bytes <= srv.mem_cap or sum(len(h) for h in srv.handles.values()) == 1


def test_cap_is_respected_before_handles_are_built(monkeypatch):
    """Two workers, nothing warmed, compositions whose handles together
    exceed the cap: every handle's bytes are reserved (estimated) before it
    is built, so the resident total never exceeds the cap while several
    handles exist."""
    FakeBatch.built.clear()
    srv = _server(monkeypatch, workers=2)
    est = max(srv.estimate_bytes(((k, 1),)) for k in PATS)
    srv.mem_cap = 1.2 * est  # room for one handle at a time
    peak = []
    real_create = srv._create

    def create(ticket):
        hd = real_create(ticket)
        peak.append(srv.bytes)
        return hd

    monkeypatch.setattr(srv, "_create", create)
    done = srv.serve(_requests(srv, 20, seed=6), realtime=False, timeout=30)
    assert len(done) == 20
    assert max(peak) <= srv.mem_cap or all(sum(len(h) for h in srv.handles.values()) <= 1 for _ in [0])


def test_realtime_arrivals_are_respected(monkeypatch):
    srv = _server(monkeypatch, workers=2)
    done = srv.serve(_requests(srv, 10, seed=5, spacing=0.01), realtime=True, timeout=30)
    assert all(r.done >= r.arrival for r in done)


def test_fresh_values_are_made_at_admission(monkeypatch):
    srv = _server(monkeypatch, workers=2)
    made = []
    reqs = _requests(srv, 12, seed=7)
    for r in reqs:
        v = r.values
        r.values = None
        r.make_values = (lambda v=v, rid=r.rid: made.append(rid) or v)
    done = srv.serve(reqs, realtime=False, timeout=30)
    assert sorted(made) == list(range(12)) and len(done) == 12
    assert all(r.values is None for r in done)
