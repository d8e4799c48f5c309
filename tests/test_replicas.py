"""The replica path for several GPUs on CPU: two gloo ranks deal queries
round-robin, search their shards (a stand-in search function, since the
index needs a GPU) and rank 0 gathers the results in input order; timings
reduce to the maximum over ranks."""
import os
import socket
import tempfile

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from topaz_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _fake_search(qs):
    # a per-query result that depends only on the query, like the real one
    return [{"len": len(q), "sum": int(np.frombuffer(q, np.uint8).sum())} for q in qs]


def _rank(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        queries = [bytes(rng.integers(65, 90, int(rng.integers(1, 40)), dtype=np.uint8)) for _ in range(23)]
        got = replicas.search_replicated(queries, _fake_search, rank, world)
        worst = replicas.max_over_ranks(1.5 + rank, world)
        if rank == 0:
            want = _fake_search(queries)
            ok = got == want and worst == 1.5 + (world - 1)
            with open(os.path.join(out_dir, "ok"), "w") as f:
                f.write("1" if ok else "0")
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_shard_covers_every_query_once():
    for n in (0, 1, 7, 23):
        for world in (1, 2, 3, 8):
            ids = np.concatenate([replicas.shard(n, r, world) for r in range(world)])
            assert sorted(ids.tolist()) == list(range(n))


def test_two_ranks_gather_in_input_order():
    with tempfile.TemporaryDirectory() as d:
        mp.spawn(_rank, args=(2, _free_port(), d), nprocs=2, join=True)
        assert open(os.path.join(d, "ok")).read() == "1"


def test_single_rank_is_the_plain_search():
    qs = [b"AB", b"C", b"DEF"]
    assert replicas.search_replicated(qs, _fake_search, 0, 1) == _fake_search(qs)
    assert replicas.max_over_ranks(2.5, 1) == 2.5
