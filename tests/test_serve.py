"""The serving loop's host logic on the CPU, with a stand-in backend:
admission by device-memory budget, batching of what waits, per-kind FIFO
order, results to the right request, failures to the batch's requests."""

import threading
import time

import numpy as np
import pytest

from rivet_prores_b200.serve import Server, poisson_run


class FakeBackend:
    """Echoes payloads after a delay; records every batch and the budget in use."""

    def __init__(self, delay=0.02, fail_on=None):
        self.delay = delay
        self.fail_on = fail_on
        self.batches = []
        self.lock = threading.Lock()
        self.server = None
        self.over_budget = False

    def _run(self, reqs, tag):
        with self.lock:
            self.batches.append([r.payload for r in reqs])
            if self.server and self.server.in_use > self.server.budget and len(reqs) > 1:
                self.over_budget = True
        if self.fail_on is not None and any(r.payload == self.fail_on for r in reqs):
            raise RuntimeError("device failure")
        time.sleep(self.delay)
        return [(tag, r.payload) for r in reqs]

    def decode(self, reqs):
        return self._run(reqs, "dec")

    def encode(self, reqs):
        return self._run(reqs, "enc")


def test_results_reach_their_requests_and_batches_form():
    be = FakeBackend(delay=0.05)
    srv = Server(be, memory_budget=1000, max_batch=8, workers=2)
    be.server = srv
    futs = [srv.submit_decode(bytes([i]), cost=10) for i in range(40)]
    futs += [srv.submit_encode(i, None, cost=10) for i in range(10)]
    for i, f in enumerate(futs[:40]):
        assert f.result(timeout=10) == ("dec", bytes([i]))
    for i, f in enumerate(futs[40:]):
        assert f.result(timeout=10) == ("enc", i)
    srv.close()
    st = srv.stats()
    assert st["requests"] == 50
    assert max(len(b) for b in be.batches) > 1
    assert all(len(b) <= 8 for b in be.batches)


def test_admission_keeps_in_flight_memory_within_budget():
    be = FakeBackend(delay=0.03)
    srv = Server(be, memory_budget=100, max_batch=64, workers=3)
    be.server = srv
    futs = [srv.submit_decode(bytes([i % 256]), cost=30) for i in range(30)]
    for f in futs:
        f.result(timeout=10)
    srv.close()
    assert srv.peak_in_use <= 100
    assert not be.over_budget
    assert all(len(b) <= 3 for b in be.batches)


def test_a_request_larger_than_the_budget_runs_alone():
    be = FakeBackend(delay=0.01)
    srv = Server(be, memory_budget=50, workers=2)
    f = srv.submit_decode(b"big", cost=500)
    g = srv.submit_decode(b"small", cost=10)
    assert f.result(timeout=10) == ("dec", b"big")
    assert g.result(timeout=10) == ("dec", b"small")
    srv.close()
    assert [b"big"] in be.batches


def test_fifo_within_a_kind():
    be = FakeBackend(delay=0.0)
    srv = Server(be, memory_budget=10_000, max_batch=4, workers=1)
    futs = [srv.submit_decode(bytes([i]), cost=1) for i in range(20)]
    for f in futs:
        f.result(timeout=10)
    srv.close()
    order = [p for b in be.batches for p in b]
    assert order == [bytes([i]) for i in range(20)]


def test_a_failing_batch_fails_its_requests_only():
    be = FakeBackend(delay=0.0, fail_on=b"\x07")
    srv = Server(be, memory_budget=10_000, max_batch=1, workers=1)
    futs = [srv.submit_decode(bytes([i]), cost=1) for i in range(10)]
    for i, f in enumerate(futs):
        if i == 7:
            with pytest.raises(RuntimeError):
                f.result(timeout=10)
        else:
            assert f.result(timeout=10) == ("dec", bytes([i]))
    srv.close()


def test_poisson_run_reports_latency_percentiles():
    be = FakeBackend(delay=0.002)
    srv = Server(be, memory_budget=10_000, max_batch=16, workers=2)
    st = poisson_run(srv, lambda i: ("decode", bytes([i % 256])), rate=400.0, seconds=0.5, seed=1)
    srv.close()
    assert st["requests"] > 100
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]


def test_pinned_pool_reuses_a_block_only_after_every_view_is_gone():
    import gc

    from rivet_prores_b200.serve import PinnedPool

    pool = PinnedPool(limit=8 << 20, allocate=lambda n: np.zeros(n, np.uint8))
    a = pool.take(1000)
    assert a.dtype == np.uint16 and a.size == 1000
    a[:] = 7
    view = a[10:20]
    del a
    gc.collect()
    b = pool.take(1000)  # the first block is still viewed: a new one
    assert pool.made == 2
    assert (view == 7).all()
    del view, b
    gc.collect()
    c = pool.take(300_000)  # the same 1 MiB class: a pooled block
    assert pool.made == 2 and c.size == 300_000
    d = pool.take(600_000)  # 1.2 MB: the 2 MiB class, a new block
    assert pool.made == 3
    del c, d
    gc.collect()
    assert pool.idle == 4 << 20


def test_pinned_pool_keeps_at_most_its_limit_idle():
    import gc

    from rivet_prores_b200.serve import PinnedPool

    pool = PinnedPool(limit=2 << 20, allocate=lambda n: np.zeros(n, np.uint8))
    xs = [pool.take(100) for _ in range(5)]
    del xs
    gc.collect()
    assert pool.idle == 2 << 20
