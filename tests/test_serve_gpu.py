"""The serving loop (continuous batching over a resident index): every
request gets the same hits in a mix of concurrent requests as alone."""
import random
import threading

import numpy as np
import pytest

from sa_util import make_db
from topaz_b200 import alphabet as ab, native, serve, synth

pytestmark = pytest.mark.gpu

BLOSUM62 = synth.matrix("BLOSUM62")
FIELDS = ("protein", "rawscore", "qend", "send", "bitscore", "evalue", "sw_status")


@pytest.fixture(scope="module")
def served():
    prot = synth.protein_db(3000, seed=41)
    qs = synth.search_queries(prot, 40, 20, seed=42, hi=3200)
    db = make_db(prot)
    queries = [native.prepare_query(ab.upper_aa(s).tobytes()) for s in qs.seqs]
    return native.Index(db), queries


def _alone(ix, qs, report):
    r = ix.search(qs, BLOSUM62, report=report)
    out = []
    for k in range(len(qs)):
        a, b = r["hit_off"][k], r["hit_off"][k + 1]
        out.append({f: r[f][a:b] for f in FIELDS})
    return out


@pytest.mark.parametrize("workers,max_batch,budget", [(2, 7, None), (3, 64, None), (2, 5, 1)])
def test_requests_same_alone_and_in_the_mix(cuda, served, workers, max_batch, budget):
    ix, queries = served
    report = {"max_evalue": 10.0}
    rng = random.Random(workers * 100 + max_batch)
    reqs = []
    i = 0
    while i < len(queries):
        n = rng.randint(1, 9)
        reqs.append(queries[i:i + n])
        i += n
    srv = serve.SearchServer(ix, BLOSUM62, workers=workers, max_batch=max_batch,
                             mem_budget=budget, report=report)
    futs = [None] * len(reqs)

    def client(idx):
        for j in idx:
            futs[j] = srv.submit(reqs[j])

    th = [threading.Thread(target=client, args=(list(range(c, len(reqs), 3)),)) for c in range(3)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    got = [f.result(timeout=300) for f in futs]
    srv.close()
    assert sum(n for n, _ in srv.batches) == len(queries)
    if max_batch < 10:
        assert len(srv.batches) >= len(queries) // max_batch
    for q, g in zip(reqs, got):
        for a, b in zip(_alone(ix, q, report), g):
            for f in FIELDS:
                assert np.array_equal(a[f], b[f]), f
    assert all(serve.latency_of(f) >= 0 for f in futs)
    assert sum(len(h["protein"]) for g in got for h in g) > 0


def test_empty_request_and_close(cuda, served):
    ix, queries = served
    srv = serve.SearchServer(ix, BLOSUM62, workers=1)
    assert srv.submit([]).result(timeout=10) == []
    srv.close()
    with pytest.raises(RuntimeError):
        srv.submit(queries[:1])
