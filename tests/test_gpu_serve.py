"""Serving loop on the GPU: requests of different patterns are merged into
one forest per admission round (fronts merged level by level) and rounds run
concurrently on several streams; every result must be the one the request
gets alone.

Bars: plain FP64 -- the served solution is bitwise equal to the same
request factored and solved alone (requests never share arithmetic);
mixed -- every request reaches backward error <= 1e-12 and agrees with its
alone solution within 1e-9 relative."""
import numpy as np
import pytest

import multifrontal as mf
from multifrontal import serve
from multifrontal import testmatrices as tm

pytestmark = pytest.mark.gpu


def _patterns():
    return {
        "g2d12": (lambda s: tm.grid_laplacian(12, 12, seed=s), "amf", 4),
        "g2d20": (lambda s: tm.grid_laplacian(20, 20, seed=s), "amf", 4),
        "g3d6": (lambda s: tm.grid_laplacian(6, 6, 6, seed=s), mf.grid_nd_order(6, 6, 6), 2),
    }


def _stream(srv, count, seed):
    rng = np.random.default_rng(seed)
    pats = _patterns()
    keys = list(pats)
    reqs, mats = [], {}
    t = 0.0
    for i in range(count):
        k = keys[rng.integers(len(keys))]
        A = pats[k][0](1000 + i)
        n = A.shape[0]
        B = tm.rhs(n, int(rng.integers(1, 5)), seed=i)
        t += rng.exponential(0.001)
        reqs.append(serve.Request(i, k, srv.lower_values(k, A), B, arrival=t))
        mats[i] = A
    return reqs, mats


def _alone(A, order, B, mixed):
    P, S = mf.symbolic(A, alg=order)
    F = mf.cholesky_(mf.ChordalCholesky(A, P, S, mixed=mixed))
    X = mf.ldiv(F, B)
    F.close()
    return X


@pytest.mark.parametrize("mixed", [False, True])
def test_served_results_equal_alone(mixed):
    srv = serve.Server(mixed=mixed, workers=3)
    for k, (gen, order, batch) in _patterns().items():
        srv.add_pattern(k, gen(0), order=order, batch=batch, size_class=0)
    srv.warm()
    reqs, mats = _stream(srv, 40, seed=7 + mixed)
    done = srv.serve(reqs, realtime=True, timeout=120)
    assert len(done) == 40 and all(r.done >= r.arrival for r in done)
    assert max(r.batch_size for r in done) > 1  # some requests really shared a round
    assert any(len(c) > 1 for c in srv.rounds)  # some round merged different patterns
    pats = _patterns()
    for r in done:
        A = mats[r.rid]
        eta = tm.backward_error(A, r.X, r.B).max()
        assert eta <= (1e-12 if mixed else 1e-13), (r.rid, eta)
        if mixed:
            assert abs(r.eta - eta) <= 1e-3 * eta + 1e-16
    for r in done[::5]:
        Xa = _alone(mats[r.rid], pats[r.key][1], r.B, mixed)
        if mixed:
            assert np.abs(Xa - r.X).max() <= 1e-9 * np.abs(Xa).max()
        else:
            assert np.array_equal(Xa, r.X), r.rid
    stats = serve.latency_stats(done)
    assert stats["p99_ms"] >= stats["p50_ms"] > 0
    srv.close()


def test_memory_cap_evicts_idle_handles():
    srv = serve.Server(mixed=False, workers=1)
    for k, (gen, order, batch) in _patterns().items():
        srv.add_pattern(k, gen(0), order=order, batch=batch, size_class=0)
    srv.warm(["g2d12"], counts=[1])
    one = srv.bytes
    assert one > 0
    srv.mem_cap = one * 1.5  # room for about one handle
    reqs, mats = _stream(srv, 12, seed=3)
    done = srv.serve(reqs, realtime=False, timeout=120)
    assert len(done) == 12
    assert srv.bytes <= max(srv.mem_cap, max(h.bytes for hs in srv.handles.values() for h in hs))
    for r in done:
        assert tm.backward_error(mats[r.rid], r.X, r.B).max() <= 1e-13
    srv.close()
