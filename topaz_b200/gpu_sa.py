"""Suffix array of a DB text on the GPU by prefix doubling (torch.sort).

Used to prepare large benchmark databases quickly; `topaz index` writes the
same array (the SA of a text is unique) with its own SA-IS on the host.
Ranks are combined into int64 keys rank*(n+2) + next_rank + 1, so texts up
to ~3e9 bytes."""
import numpy as np


def suffix_array(T: np.ndarray, device="cuda") -> np.ndarray:
    import torch
    n = len(T)
    if n == 0:
        return np.zeros(0, np.int64)
    if n > 3_000_000_000:
        raise ValueError("text too long for int64 rank keys")
    rank = torch.from_numpy(np.ascontiguousarray(T)).to(device).long()
    k = 1
    while True:
        nxt = torch.full_like(rank, -1)
        if k < n:
            nxt[: n - k] = rank[k:]
        key = rank * (n + 2) + (nxt + 1)
        del nxt
        skey, sa = torch.sort(key)
        del key
        step = torch.ones_like(skey)
        step[0] = 0
        step[1:] = (skey[1:] != skey[:-1]).long()
        del skey
        newr = torch.cumsum(step, 0)
        del step
        rank = torch.empty_like(newr)
        rank[sa] = newr
        if int(newr[-1]) == n - 1:
            return sa.cpu().numpy()
        del newr
        k *= 2
