"""The oracle (CPU restatement) against the reference's golden vectors and,
when oracle/_ref is built, against the live reference on fresh cases."""
import ctypes

import numpy as np
import pytest

import oracle
from topaz_b200 import dbformat, synth, alphabet as ab


def _golden_settings(g):
    for k in g:
        if k.count("_") == 2 and not k.startswith("mat_"):
            name, go, ge = k.split("_")
            yield k, g["mat_" + name], int(go), int(ge)


def test_oracle_sw_matches_golden(golden_sw):
    g = golden_sw
    n = 0
    for key, mat, go, ge in _golden_settings(g):
        got = np.stack(oracle.oracle_sw(g["q"], g["qoff"], g["qlen"], g["s"], g["soff"],
                                        g["slen"], mat, go, ge))
        bad = np.flatnonzero((got != g[key]).any(axis=0))
        assert bad.size == 0, (key, bad[:5], got[:, bad[:5]], g[key][:, bad[:5]])
        n += 1
    assert n == 5


def test_golden_covers_overflow_paths(golden_sw):
    ref = golden_sw["BLOSUM62_11_1"]
    assert (ref[0] >= 251).sum() > 50          # u8 saturation -> i16 rerun
    assert (ref[0] == 0).sum() > 5             # no positive cell
    assert (golden_sw["qlen"] == 1).sum() > 0


def _golden_db(g):
    ind = g["ind"].view(dbformat.IND_DTYPE)
    return dbformat.Database(g["T"], g["SA"].astype(np.int64), ind, g["headers"].tobytes())


@pytest.mark.parametrize("variant", ["default", "tight"])
def test_oracle_search_matches_golden(golden_search, variant):
    g = golden_search
    db = _golden_db(g)
    mat = synth.matrix("BLOSUM62")
    seeds, aligns = (int(x) for x in g["seeds_" + variant])
    opts = oracle.Opts(100, 1e-3, 11, 1, 0.267, 0.041, 0.14, 5, seeds, aligns)
    popn = g["popn_" + variant]
    pops = g["pops_" + variant]
    meta = g["meta_" + variant]
    hi, hf = g["hitsi_" + variant], g["hitsf_" + variant]
    p0 = h0 = 0
    for qi in range(len(g["qlen"])):
        q = g["qcat"][g["qoff"][qi]:g["qoff"][qi] + g["qlen"][qi]].tobytes()
        P, hits, npops, ncnt, nh = oracle.oracle_query(db, q, mat, opts)
        assert (npops, ncnt, nh) == tuple(meta[qi])
        ref = pops[:, p0:p0 + popn[qi]]
        p0 += popn[qi]
        mine = np.stack([P["row"], P["off"], P["score"], P["len"], P["counted"]])[:, :popn[qi]]
        assert (mine == ref).all()
        rh = hi[h0:h0 + nh]
        rf = hf[h0:h0 + nh]
        h0 += nh
        mh = np.array([(x.db_index, x.gapless_score, x.is_aligned, x.rawscore, x.qend, x.send)
                       for x in hits], np.int64).reshape(-1, 6)
        al = rh[:, 2] == 1
        assert (mh[:, :3] == rh[:, :3]).all()
        assert (mh[al, 3:] == rh[al, 3:]).all()
        mf = np.array([(x.evalue, x.bitscore) for x in hits]).reshape(-1, 2)
        assert (mf[al] == rf[al]).all()          # bit-identical doubles


needs_ref = pytest.mark.skipif(oracle.libref() is None, reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("go,ge,name", [(11, 1, "BLOSUM62"), (7, 2, "BLOSUM50"), (10, 1, "PAM70")])
def test_oracle_sw_matches_live_reference(go, ge, name):
    ps = synth.sw_pairs(1200, seed=go * 100 + ge, q_range=(1, 1024), s_range=(1, 3000))
    mat = synth.matrix(name)
    a = np.stack(oracle.reference_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, go, ge))
    b = np.stack(oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, go, ge))
    assert (a == b).all()


@needs_ref
def test_oracle_seeds_and_walk_match_live_reference():
    L = oracle.libref()
    prot = synth.protein_db(1500, seed=77)
    qs = synth.search_queries(prot, 5, 2, seed=78)
    db = dbformat.build_from_records([(p.encode(), s) for p, s in zip(prot.ids, prot.seqs)])
    SA = np.zeros(db.Tsize, np.int64)
    assert L.divsufsort64(oracle._p(db.T), oracle._p(SA), ctypes.c_int64(db.Tsize)) == 0
    db.SA = SA
    h = L.ref_db_open(oracle._p(db.T), ctypes.c_uint64(db.Tsize), oracle._p(SA),
                      oracle._p(db.ind), ctypes.c_uint64(db.Psize), db.headers,
                      ctypes.c_uint64(len(db.headers)))
    orc = oracle.liboracle()
    mat = synth.matrix("BLOSUM62")
    try:
        for s in qs.seqs:
            qi = ab.aa_to_internal(s).tobytes()
            n = len(qi) - 5
            arrs = [np.zeros(n, np.int64)] + [np.zeros(n, np.int32) for _ in range(4)]
            L.ref_seed_list(ctypes.c_void_p(h), qi, len(qi), 5, b"BLOSUM62",
                            *[oracle._p(a) for a in arrs])
            for i in range(n):
                if arrs[0][i] == -2:
                    continue
                lb = orc.orc_lower_bound(oracle._p(db.T), ctypes.c_int64(db.Tsize), oracle._p(SA),
                                         qi[i:], ctypes.c_int64(len(qi) - i))
                assert lb == arrs[0][i]
            opts = oracle.Opts(100, 1e-3, 11, 1, 0.267, 0.041, 0.14, 5, 2000, 200)
            P, hits, npops, ncnt, nh = oracle.oracle_query(db, qi, mat, opts)
            MAXP = 1 << 16
            rows = np.zeros(MAXP, np.int64)
            arr = [np.zeros(MAXP, np.int32) for _ in range(4)]
            rn, rc = ctypes.c_int64(), ctypes.c_int64()
            hb = (oracle.RHit * 6000)()
            rnh = L.ref_query_run(ctypes.c_void_p(h), qi, len(qi), b"BLOSUM62", 100,
                                  ctypes.c_double(1e-3), 11, 1, ctypes.c_double(0.267),
                                  ctypes.c_double(0.041), ctypes.c_double(0.14), 5, 2000, 200, 1,
                                  oracle._p(rows), *[oracle._p(a) for a in arr],
                                  ctypes.c_int64(MAXP), ctypes.byref(rn), ctypes.byref(rc), hb, 6000)
            assert (rn.value, rc.value, rnh) == (npops, ncnt, nh)
            m = min(npops, MAXP)
            assert (rows[:m] == P["row"][:m]).all() and (arr[1][:m] == P["score"][:m]).all()
            for x, y in zip(hb[:rnh], hits):
                assert (x.db_index, x.gapless_score, x.is_aligned) == (y.db_index, y.gapless_score, y.is_aligned)
                if x.is_aligned:
                    assert (x.rawscore, x.qend, x.send, x.evalue) == (y.rawscore, y.qend, y.send, y.evalue)
    finally:
        L.ref_db_close(ctypes.c_void_p(h))
