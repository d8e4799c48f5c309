"""Generates the golden fixtures in tests/golden/ by running the UNMODIFIED
reference (compiled into oracle/_ref by `make -C oracle ref`).

    python tests/golden/make_golden.py

The reference ships no tests or fixtures of its own; these vectors are its
outputs on seeded synthetic inputs:

* sw_golden.npz     -- ssw_init + ssw_align on pairs (several matrices and
                       gap settings) incl. short/degenerate edge pairs;
* search_golden.npz -- a small DB (T, .ind, SA from the reference's
                       divsufsort64) with per-query reference results: the
                       pop sequence of the best-first walk, the hitlist in
                       traversal order with SW scores/ends/E-values.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from topaz_b200 import dbformat, synth, alphabet as ab  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
SW_SETTINGS = [("BLOSUM62", 11, 1), ("BLOSUM62", 3, 1), ("BLOSUM45", 13, 3), ("PAM30", 9, 1),
               ("BLOSUM80", 10, 1)]


def edge_pairs(rng):
    qs, ss = [], []
    for ql in (1, 2, 3, 15, 16, 17, 31, 32, 33, 63, 64, 65):
        for sl in (0, 1, 2, 7, 40):
            qs.append(rng.integers(0, 25, ql).astype(np.int8))
            ss.append(rng.integers(0, 25, sl).astype(np.int8))
    for ql in (1, 20, 100):                        # all X: score 0
        qs.append(np.full(ql, 23, np.int8)); ss.append(np.full(50, 23, np.int8))
    for ql in (5, 64, 300, 1000, 1024):            # identical: deep u8 overflow
        q = rng.integers(0, 20, ql).astype(np.int8)
        qs.append(q); ss.append(q.copy())
    for ql in (1000, 1024):                        # W-rich: large i16 scores
        q = np.full(ql, ab.MATRIX_ORDER.index("W"), np.int8)
        qs.append(q); ss.append(np.concatenate([q, q[:100]]))
    return qs, ss


def pack(seqs):
    lens = np.array([len(x) for x in seqs], np.int32)
    off = np.zeros(len(seqs), np.int64)
    off[1:] = np.cumsum(lens)[:-1]
    return (np.concatenate(seqs) if len(seqs) else np.zeros(0, np.int8)), off, lens


def make_sw():
    rng = np.random.default_rng(1234)
    ps = synth.sw_pairs(1500, seed=101, q_median=150, q_range=(1, 1024), s_median=180,
                        s_range=(1, 1500))
    qs = [ps.q[o:o + l] for o, l in zip(ps.qoff, ps.qlen)]
    ss = [ps.s[o:o + l] for o, l in zip(ps.soff, ps.slen)]
    eq, es = edge_pairs(rng)
    q, qoff, qlen = pack(qs + eq)
    s, soff, slen = pack(ss + es)
    res = {"q": q, "qoff": qoff, "qlen": qlen, "s": s, "soff": soff, "slen": slen}
    L = oracle.libref()
    for name, go, ge in SW_SETTINGS:
        mat = np.ctypeslib.as_array(L.ref_matrix(name.encode()), shape=(625,)).copy()
        sc, re, rd, stt = oracle.reference_sw(q, qoff, qlen, s, soff, slen, mat, go, ge)
        key = "%s_%d_%d" % (name, go, ge)
        res[key] = np.stack([sc, re, rd, stt]).astype(np.int32)
        res["mat_" + name] = mat
    np.savez_compressed(os.path.join(OUT, "sw_golden.npz"), **res)


SEARCH_VARIANTS = [("default", 300000, 5000), ("tight", 300, 50)]


def make_search():
    prot = synth.protein_db(400, seed=201)
    qs = synth.search_queries(prot, 8, 2, seed=202)
    db = dbformat.build_from_records([(p.encode(), s) for p, s in zip(prot.ids, prot.seqs)])
    L = oracle.libref()
    SA = np.zeros(db.Tsize, np.int64)
    assert L.divsufsort64(oracle._p(db.T), oracle._p(SA), ctypes.c_int64(db.Tsize)) == 0
    h = L.ref_db_open(oracle._p(db.T), ctypes.c_uint64(db.Tsize), oracle._p(SA),
                      oracle._p(db.ind), ctypes.c_uint64(db.Psize), db.headers,
                      ctypes.c_uint64(len(db.headers)))
    res = {"T": db.T, "SA": SA.astype(np.int32), "ind": db.ind.view(np.uint8),
           "headers": np.frombuffer(db.headers, np.uint8)}
    qints = [ab.aa_to_internal(s).tobytes() for s in qs.seqs]
    qcat, qoff, qlen = pack([np.frombuffer(x, np.int8) for x in qints])
    res.update(qcat=qcat, qoff=qoff, qlen=qlen)
    MAXP = 4000
    for vname, seeds, aligns in SEARCH_VARIANTS:
        pops, hits, meta = [], [], []
        for qi in qints:
            rows = np.zeros(MAXP, np.int64)
            arr = [np.zeros(MAXP, np.int32) for _ in range(4)]
            npops, ncnt = ctypes.c_int64(), ctypes.c_int64()
            hb = (oracle.RHit * 6000)()
            nh = L.ref_query_run(ctypes.c_void_p(h), qi, len(qi), b"BLOSUM62", 100,
                                 ctypes.c_double(1e-3), 11, 1, ctypes.c_double(0.267),
                                 ctypes.c_double(0.041), ctypes.c_double(0.14), 5, seeds, aligns,
                                 1, oracle._p(rows), *[oracle._p(a) for a in arr],
                                 ctypes.c_int64(MAXP), ctypes.byref(npops), ctypes.byref(ncnt),
                                 hb, 6000)
            n = min(npops.value, MAXP)
            pops.append(np.stack([rows[:n], arr[0][:n], arr[1][:n], arr[2][:n], arr[3][:n]]))
            hits.append(np.array([(x.db_index, x.gapless_score, x.is_aligned, x.rawscore, x.qend,
                                   x.send) for x in hb[:nh]], np.int64).reshape(-1, 6))
            hits.append(np.array([(x.evalue, x.bitscore) for x in hb[:nh]], np.float64).reshape(-1, 2))
            meta.append((npops.value, ncnt.value, nh))
        res["pops_" + vname] = np.concatenate([p for p in pops], axis=1)
        res["popn_" + vname] = np.array([p.shape[1] for p in pops], np.int64)
        res["hitsi_" + vname] = np.concatenate(hits[0::2])
        res["hitsf_" + vname] = np.concatenate(hits[1::2])
        res["meta_" + vname] = np.array(meta, np.int64)
        res["seeds_" + vname] = np.array([seeds, aligns], np.int64)
    L.ref_db_close(ctypes.c_void_p(h))
    np.savez_compressed(os.path.join(OUT, "search_golden.npz"), **res)


if __name__ == "__main__":
    if oracle.libref() is None and not oracle.build_ref():
        sys.exit("the reference sources are needed to regenerate the fixtures")
    make_sw()
    make_search()
    for f in ("sw_golden.npz", "search_golden.npz"):
        print(f, os.path.getsize(os.path.join(OUT, f)))
