"""Search serving: a continuous-batching request loop over a resident index.

Requests (lists of queries, internal alphabet after SEG, as
``native.prepare_query`` makes them) arrive through ``submit``.  Worker
threads -- each one a host thread with its own CUDA default stream, so their
batches run on the device at the same time -- take every waiting query, in
arrival order and across request boundaries, up to ``max_batch`` queries and
up to the device memory still free under ``mem_budget``, run them through
``tpz_search_batch`` in report mode, and hand each query's reported hits back
to its request.  A request completes when its last query is back; a request
that arrives while others are on the GPU is admitted as soon as a worker and
memory are free, so short requests are not held behind long ones.

Each query's result does not depend on the queries batched with it (every
query has its own walk, hitlist and SW pairs), so a request gets the same
hits alone and in a mix; the tests check exactly that.
"""
from __future__ import annotations

import collections
import threading
import time
from concurrent.futures import Future

import numpy as np

from . import native


def query_device_bytes(qlen: int, num_hits: int = 100, alignments: int = 5000,
                       min_hit_length: int = 5) -> int:
    """Upper estimate of the device memory one query takes inside
    tpz_search_batch, from the library itself
    (tpz_search_query_device_bytes: the same capacities the batch sizes its
    buffers by)."""
    return native.query_device_bytes(qlen, num_hits=num_hits, alignments=alignments,
                                     min_hit_length=min_hit_length)


class _Request:
    __slots__ = ("queries", "results", "left", "future", "t_submit", "t_done", "cancelled")

    def __init__(self, queries):
        self.queries = queries
        self.results = [None] * len(queries)
        self.left = len(queries)
        self.future = Future()
        self.t_submit = time.perf_counter()
        self.t_done = None
        self.cancelled = False


class SearchServer:
    """Continuous batching of search requests over one resident ``Index``."""

    def __init__(self, index, mat, workers: int = 2, max_batch: int = 2000,
                 mem_budget: int | None = None, report=None, search_kwargs=None):
        self.ix = index
        self.mat = np.ascontiguousarray(mat, dtype=np.int8)
        self.max_batch = int(max_batch)
        self.report = dict(report or {"max_evalue": 1e-3})
        self.kw = dict(search_kwargs or {})
        if mem_budget is None:
            import torch
            free, _ = torch.cuda.mem_get_info()
            mem_budget = int(0.8 * free)
        self.mem_budget = int(mem_budget)
        self._mem_used = 0
        self._pending = collections.deque()     # (request, query index)
        self._cv = threading.Condition()
        self._closed = False
        self.batches = []                       # (n queries, seconds) per finished batch
        self._threads = [threading.Thread(target=self._work, daemon=True) for _ in range(workers)]
        for t in self._threads:
            t.start()

    # -- client side
    def submit(self, queries) -> Future:
        """Queues a request; the future resolves to a list with, per query,
        a dict of its reported hits (protein, rawscore, qend, send, bitscore,
        evalue, sw_status, status)."""
        req = _Request(list(queries))
        req.future.request = req
        if not req.queries:
            req.t_done = req.t_submit
            req.future.set_result([])
            return req.future
        with self._cv:
            if self._closed:
                raise RuntimeError("server is closed")
            for i in range(len(req.queries)):
                self._pending.append((req, i))
            self._cv.notify_all()
        return req.future

    def cancel(self, future) -> bool:
        """Cancels a request: its queries still waiting are dropped, a batch
        already holding some of them finishes without handing them back, and
        the future ends cancelled.  False when the request had completed."""
        req = future.request
        with self._cv:
            if req.future.done():
                return False
            req.cancelled = True
            self._pending = collections.deque(x for x in self._pending if x[0] is not req)
            req.t_done = time.perf_counter()
            ok = req.future.cancel()
            self._cv.notify_all()
        return ok

    def close(self):
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()

    # -- worker side
    def _take(self):
        """The next batch: waiting queries in arrival order, as many as fit
        max_batch and the free part of the memory budget (at least one)."""
        with self._cv:
            while True:
                if self._pending:
                    batch, need = [], 0
                    while self._pending and len(batch) < self.max_batch:
                        req, i = self._pending[0]
                        b = query_device_bytes(len(req.queries[i]), **self._size_kw())
                        if batch and self._mem_used + need + b > self.mem_budget:
                            break
                        if not batch and self._mem_used + b > self.mem_budget and self._mem_used:
                            break                   # wait for memory to come back
                        self._pending.popleft()
                        batch.append((req, i))
                        need += b
                    if batch:
                        self._mem_used += need
                        return batch, need
                if self._closed:
                    return None, 0
                self._cv.wait()

    def _size_kw(self):
        kw = {k: self.kw[k] for k in ("num_hits", "alignments", "min_hit_length") if k in self.kw}
        return kw

    def _work(self):
        while True:
            batch, need = self._take()
            if batch is None:
                return
            t0 = time.perf_counter()
            try:
                r = self.ix.search([req.queries[i] for req, i in batch], self.mat,
                                   report=self.report, **self.kw)
                err = None
            except Exception as e:              # hand the failure to every request
                r, err = None, e
            dt = time.perf_counter() - t0
            done = []
            with self._cv:
                self._mem_used -= need
                self.batches.append((len(batch), dt))
                for k, (req, i) in enumerate(batch):
                    if req.cancelled:
                        continue
                    if err is not None:
                        if not req.future.done():
                            req.t_done = time.perf_counter()
                            req.future.set_exception(err)
                        continue
                    a, b = r["hit_off"][k], r["hit_off"][k + 1]
                    req.results[i] = {f: r[f][a:b] for f in ("protein", "rawscore", "qend", "send",
                                                              "bitscore", "evalue", "sw_status")}
                    req.results[i]["status"] = int(r["status"][k])
                    req.left -= 1
                    if req.left == 0:
                        req.t_done = time.perf_counter()
                        done.append(req)
                self._cv.notify_all()
            for req in done:
                req.future.set_result(req.results)


def latency_of(future) -> float:
    """Seconds from submit to completion of a finished request."""
    req = future.request
    return req.t_done - req.t_submit


def saturated_qps(index, mat, queries, workers: int, max_batch: int, report=None,
                  request_size: int = 250) -> float:
    """Queries per second the serving loop delivers with every request
    already waiting (its capacity on this query mix)."""
    srv = SearchServer(index, mat, workers=workers, max_batch=max_batch, report=report)
    try:
        srv.submit(queries[:min(len(queries), 50)]).result()          # warm-up
        t0 = time.perf_counter()
        futs = [srv.submit(queries[i:i + request_size])
                for i in range(0, len(queries), request_size)]
        for f in futs:
            f.result()
        return len(queries) / (time.perf_counter() - t0)
    finally:
        srv.close()


def autotune(index, mat, queries, report=None,
             candidates=((2, 1000), (2, 2000), (3, 1000), (3, 2000), (4, 1000), (4, 2000),
                         (3, 3000))):
    """Picks the worker count and batch cap of the serving loop for this
    index and query mix: the candidate with the highest saturated
    throughput on `queries` (a sample of the expected requests).  Returns
    ((workers, max_batch), {candidate: queries/s})."""
    seen = {}
    for w, b in candidates:
        seen[(w, b)] = saturated_qps(index, mat, queries, w, b, report=report)
    best = max(seen, key=seen.get)
    return best, seen

