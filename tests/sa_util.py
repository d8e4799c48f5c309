"""Suffix arrays for test databases (prefix doubling in numpy; small texts).

Test infrastructure: the order is plain byte-wise lexicographic with a
suffix that is a proper prefix of another sorting first -- the SA that
divsufsort64 writes for `topaz index` (the SA of a text is unique)."""
import numpy as np


def suffix_array(T: np.ndarray) -> np.ndarray:
    n = len(T)
    rank = T.astype(np.int64)
    k = 1
    while True:
        r2 = np.full(n, -1, dtype=np.int64)
        if k < n:
            r2[: n - k] = rank[k:]
        key = rank * (n + 300) + (r2 + 1)
        sa = np.argsort(key, kind="stable")
        sk = key[sa]
        newrank = np.empty(n, dtype=np.int64)
        newrank[sa] = np.concatenate([[0], np.cumsum(sk[1:] != sk[:-1])])
        rank = newrank
        if n == 0 or rank[sa[-1]] == n - 1:
            return sa.astype(np.int64)
        k *= 2


def make_db(prot):
    from topaz_b200 import dbformat
    db = dbformat.build_from_records([(p.encode(), s) for p, s in zip(prot.ids, prot.seqs)])
    db.SA = suffix_array(db.T)
    return db
