"""Several GPUs: one full replica of the resident index per GPU, queries
dealt out round-robin, results gathered back in input order.

The search shards by query only: every rank holds the whole index (seed
lookup, walk, hitlist and SW of a query touch nothing but read-only index
data and that query's own state), so no collective is needed on the data
path.  Sharding the database instead would change results (the walk's
best-first order, capacity eviction and -S counting are global per query).
The only collectives are the gathering of results and of timings, over
``torch.distributed`` (NCCL between GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

import numpy as np


def shard(n: int, rank: int, world: int) -> np.ndarray:
    """Indices of the queries rank `rank` searches: i with i % world == rank."""
    return np.arange(rank, n, world, dtype=np.int64)


def search_replicated(queries, search_fn, rank: int, world: int, group=None):
    """Runs `search_fn(list of queries) -> list of per-query results` on this
    rank's shard and gathers every rank's results on rank 0 in input order.
    Returns the full list on rank 0 and None elsewhere (world == 1: the
    plain result)."""
    import torch.distributed as dist
    idx = shard(len(queries), rank, world)
    mine = search_fn([queries[i] for i in idx]) if len(idx) else []
    if len(mine) != len(idx):
        raise ValueError("search_fn returned %d results for %d queries" % (len(mine), len(idx)))
    if world == 1:
        return list(mine)
    parts = [None] * world if rank == 0 else None
    dist.gather_object((idx.tolist(), list(mine)), parts, dst=0, group=group)
    if rank != 0:
        return None
    out = [None] * len(queries)
    for ids, res in parts:
        for i, r in zip(ids, res):
            out[i] = r
    return out


def max_over_ranks(x: float, world: int, device=None) -> float:
    """The largest x over all ranks (a time measured on every rank)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def index_results(r, n):
    """Per-query pieces of an Index.search result dict (report mode)."""
    out = []
    for k in range(n):
        a, b = int(r["hit_off"][k]), int(r["hit_off"][k + 1])
        out.append({f: r[f][a:b] for f in ("protein", "rawscore", "qend", "send", "bitscore",
                                           "evalue", "sw_status")})
    return out
