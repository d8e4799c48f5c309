"""The serving loop's host logic on CPU: a stand-in index (the real one needs
a GPU) records every batch, so the tests check what SearchServer promises --
per-query results independent of how queries were batched, batches in
arrival order across request boundaries, admission by the memory budget,
failures handed to the requests of the failing batch."""
import threading
import time

import numpy as np
import pytest

from topaz_b200 import serve

FIELDS = ("protein", "rawscore", "qend", "send", "bitscore", "evalue", "sw_status")


class FakeIndex:
    """search() returns, per query, len(query) % 3 hits derived from its bytes."""

    def __init__(self, delay=0.0, fail_on=None):
        self.delay, self.fail_on = delay, fail_on
        self.batches = []
        self.in_flight = 0
        self.peak = 0
        self.lock = threading.Lock()

    @staticmethod
    def hits_of(q):
        n = len(q) % 3
        base = int(np.frombuffer(q, np.uint8).sum())
        return {"protein": np.arange(n, dtype=np.int32) + base, "rawscore": np.full(n, len(q), np.int32),
                "qend": np.full(n, len(q) - 1, np.int32), "send": np.arange(n, dtype=np.int32),
                "bitscore": np.full(n, base / 7.0), "evalue": np.full(n, 1e-5),
                "sw_status": np.zeros(n, np.int32)}

    def search(self, queries, mat, report=None, **kw):
        need = sum(serve.query_device_bytes(len(q)) for q in queries)
        with self.lock:
            self.batches.append(list(queries))
            self.in_flight += need
            self.peak = max(self.peak, self.in_flight)
        try:
            time.sleep(self.delay)
            if self.fail_on is not None and any(self.fail_on in q for q in queries):
                raise RuntimeError("device error")
            per = [self.hits_of(q) for q in queries]
            out = {f: np.concatenate([p[f] for p in per]) for f in FIELDS}
            out["hit_off"] = np.concatenate([[0], np.cumsum([len(p["protein"]) for p in per])])
            out["status"] = np.zeros(len(queries), np.int32)
            return out
        finally:
            with self.lock:
                self.in_flight -= need


def _queries(rng, n, lo=30, hi=400):
    return [bytes(rng.integers(65, 90, int(rng.integers(lo, hi)), dtype=np.uint8)) for _ in range(n)]


def _same(res, qs):
    assert len(res) == len(qs)
    for r, q in zip(res, qs):
        want = FakeIndex.hits_of(q)
        for f in FIELDS:
            assert np.array_equal(r[f], want[f])
        assert r["status"] == 0


def test_results_do_not_depend_on_batching():
    rng = np.random.default_rng(3)
    ix = FakeIndex(delay=0.01)
    srv = serve.SearchServer(ix, np.zeros((25, 25), np.int8), workers=2, max_batch=7,
                             mem_budget=1 << 40)
    reqs = [_queries(rng, int(rng.integers(0, 20))) for _ in range(12)]
    futs = [srv.submit(r) for r in reqs]
    try:
        for f, r in zip(futs, reqs):
            _same(f.result(timeout=30), r)
            assert serve.latency_of(f) >= 0
    finally:
        srv.close()
    assert max(len(b) for b in ix.batches) <= 7
    # every query went to the index exactly once, some batched with others
    flat = [q for b in ix.batches for q in b]
    assert sorted(flat) == sorted(q for r in reqs for q in r)
    assert any(len(b) > 1 for b in ix.batches)


def test_one_worker_takes_queries_in_arrival_order():
    rng = np.random.default_rng(7)
    ix = FakeIndex(delay=0.005)
    srv = serve.SearchServer(ix, np.zeros((25, 25), np.int8), workers=1, max_batch=5,
                             mem_budget=1 << 40)
    reqs = [_queries(rng, int(rng.integers(1, 9))) for _ in range(8)]
    try:
        futs = [srv.submit(r) for r in reqs]
        for f, r in zip(futs, reqs):
            _same(f.result(timeout=30), r)
    finally:
        srv.close()
    assert [q for b in ix.batches for q in b] == [q for r in reqs for q in r]
    assert all(len(b) <= 5 for b in ix.batches)


def test_memory_budget_bounds_queries_in_flight():
    rng = np.random.default_rng(4)
    qs = _queries(rng, 40, 200, 300)
    one = max(serve.query_device_bytes(len(q)) for q in qs)
    budget = 3 * one
    ix = FakeIndex(delay=0.02)
    srv = serve.SearchServer(ix, np.zeros((25, 25), np.int8), workers=4, max_batch=100,
                             mem_budget=budget)
    try:
        _same(srv.submit(qs).result(timeout=60), qs)
    finally:
        srv.close()
    assert ix.peak <= budget
    assert max(len(b) for b in ix.batches) <= 3


def test_query_larger_than_the_budget_runs_alone():
    rng = np.random.default_rng(5)
    big = _queries(rng, 1, 2000, 2001)
    small = _queries(rng, 5)
    budget = serve.query_device_bytes(len(big[0])) // 2
    ix = FakeIndex(delay=0.01)
    srv = serve.SearchServer(ix, np.zeros((25, 25), np.int8), workers=3, max_batch=10,
                             mem_budget=budget)
    try:
        f1, f2 = srv.submit(big), srv.submit(small)
        _same(f1.result(timeout=30), big)
        _same(f2.result(timeout=30), small)
    finally:
        srv.close()
    assert [big[0]] in ix.batches


def test_failure_reaches_the_requests_of_the_failing_batch():
    rng = np.random.default_rng(6)
    good = _queries(rng, 4)
    bad = good[:1] + [b"POISON" + good[1]]
    ix = FakeIndex(fail_on=b"POISON")
    srv = serve.SearchServer(ix, np.zeros((25, 25), np.int8), workers=1, max_batch=1,
                             mem_budget=1 << 40)
    try:
        fb = srv.submit(bad)
        with pytest.raises(RuntimeError, match="device error"):
            fb.result(timeout=30)
        _same(srv.submit(good).result(timeout=30), good)     # the server keeps serving
    finally:
        srv.close()


def test_empty_request_and_closed_server():
    srv = serve.SearchServer(FakeIndex(), np.zeros((25, 25), np.int8), workers=1, mem_budget=1 << 30)
    assert srv.submit([]).result(timeout=5) == []
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit([b"ACDE"])


def test_device_bytes_grow_with_query_length_and_capacity():
    assert serve.query_device_bytes(100) < serve.query_device_bytes(1000)
    assert serve.query_device_bytes(500, alignments=1500) < serve.query_device_bytes(500, alignments=5000)
    # long queries (> 3000) hold 1.5 x H hits, not -A
    assert serve.query_device_bytes(3001, num_hits=100) < serve.query_device_bytes(3000, num_hits=100) * 1.2


def test_cancel_drops_waiting_queries_and_spares_other_requests():
    rng = np.random.default_rng(31)
    ix = FakeIndex(delay=0.05)
    srv = serve.SearchServer(ix, np.zeros((25, 25), np.int8), workers=1, max_batch=10,
                             mem_budget=1 << 40)
    try:
        big = _queries(rng, 200)
        small = _queries(rng, 5)
        f_big = srv.submit(big)
        f_small = srv.submit(small)
        time.sleep(0.02)                   # the first batch of the big request is running
        assert srv.cancel(f_big)
        assert f_big.cancelled()
        res = f_small.result(timeout=10)
        _same(res, small)
        seen = sum(len(b) for b in ix.batches)
        assert seen < len(big)             # most of the big request never reached the index
        assert not srv.cancel(f_small)     # already done
    finally:
        srv.close()
