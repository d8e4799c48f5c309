"""GPU parity of the search path (seed lookup, sa_hsp, best-first walk,
hitlist, SW of hits) through the C ABI, against the reference's golden
outputs and the oracle."""
import numpy as np
import pytest

import oracle
from sa_util import make_db, suffix_array
from topaz_b200 import alphabet as ab, dbformat, native, synth

pytestmark = pytest.mark.gpu

BLOSUM62 = synth.matrix("BLOSUM62")


def _golden_db(g):
    ind = g["ind"].view(dbformat.IND_DTYPE)
    return dbformat.Database(g["T"], g["SA"].astype(np.int64), ind, g["headers"].tobytes())


def _queries(g):
    return [g["qcat"][o:o + l].tobytes() for o, l in zip(g["qoff"], g["qlen"])]


@pytest.mark.parametrize("variant", ["default", "tight"])
def test_search_matches_reference_golden(cuda, golden_search, variant):
    g = golden_search
    db = _golden_db(g)
    ix = native.Index(db)
    seeds, aligns = (int(x) for x in g["seeds_" + variant])
    qs = _queries(g)
    r = ix.search(qs, BLOSUM62, seeds=seeds, alignments=aligns, trace_pops=4000)
    meta, popn, pops = g["meta_" + variant], g["popn_" + variant], g["pops_" + variant]
    hi, hf = g["hitsi_" + variant], g["hitsf_" + variant]
    p0 = h0 = 0
    db_size, nprot = db.Tsize - db.Psize, db.Psize
    for q in range(len(qs)):
        npops, ncnt, nh = meta[q]
        assert (r["npops"][q], r["ncounted"][q], r["hit_off"][q + 1] - r["hit_off"][q]) == (npops, ncnt, nh)
        n = popn[q]
        mine = np.stack([r["trace_row"][q, :n], r["trace_off"][q, :n], r["trace_score"][q, :n],
                         r["trace_len"][q, :n], r["trace_counted"][q, :n]])
        assert (mine == pops[:, p0:p0 + n]).all()
        p0 += n
        a, b = r["hit_off"][q], r["hit_off"][q + 1]
        ref = hi[h0:h0 + nh]
        reff = hf[h0:h0 + nh]
        h0 += nh
        assert (r["protein"][a:b] == ref[:, 0]).all()
        assert (r["gapless_score"][a:b] == ref[:, 1]).all()
        aligned = np.isin(r["sw_status"][a:b], [native.TPZ_SW_OK, 3])
        assert (aligned == (ref[:, 2] == 1)).all()
        sw = r["sw_status"][a:b] == native.TPZ_SW_OK
        assert (r["rawscore"][a:b][sw] == ref[sw, 3]).all()
        assert (r["qend"][a:b][sw] == ref[sw, 4]).all()
        assert (r["send"][a:b][sw] == ref[sw, 5]).all()
        for j in np.flatnonzero(sw):
            bits, ev = native.karlin(len(qs[q]), db_size, nprot, int(r["rawscore"][a + j]))
            assert ev == reff[j, 0] and bits == reff[j, 1]


@pytest.fixture(scope="module")
def fresh():
    prot = synth.protein_db(3000, seed=31)
    qs = synth.search_queries(prot, 24, 6, seed=32, hi=2600)
    db = make_db(prot)
    return db, [ab.aa_to_internal(s).tobytes() for s in qs.seqs]


@pytest.mark.parametrize("seeds,aligns", [(300000, 5000), (100000, 1500), (500, 40), (2000, 7)])
def test_search_matches_oracle(cuda, fresh, seeds, aligns):
    db, qs = fresh
    ix = native.Index(db)
    r = ix.search(qs, BLOSUM62, seeds=seeds, alignments=aligns, trace_pops=1 << 15)
    opts = oracle.Opts(100, 1e-3, 11, 1, 0.267, 0.041, 0.14, 5, seeds, aligns)
    for q, qi in enumerate(qs):
        P, hits, npops, ncnt, nh = oracle.oracle_query(db, qi, BLOSUM62, opts)
        assert nh >= 0
        assert (r["npops"][q], r["ncounted"][q]) == (npops, ncnt)
        n = min(npops, 1 << 15)
        assert (r["trace_row"][q, :n] == P["row"][:n]).all()
        assert (r["trace_score"][q, :n] == P["score"][:n]).all()
        assert (r["trace_counted"][q, :n] == P["counted"][:n]).all()
        a, b = r["hit_off"][q], r["hit_off"][q + 1]
        assert b - a == nh
        for j, h in enumerate(hits):
            k = a + j
            assert (r["protein"][k], r["gapless_score"][k]) == (h.db_index, h.gapless_score)
            if h.gapless_score >= 40:
                assert r["sw_status"][k] == h.status
                if h.status == 0:
                    assert (r["rawscore"][k], r["qend"][k], r["send"][k]) == (h.rawscore, h.qend, h.send)


@pytest.mark.parametrize("num_hits,evalue,k", [(100, 1e-3, 0.041), (7, 10.0, 0.041),
                                                (400, 2000.0, 0.041), (1, 1e-30, 0.041),
                                                (50, 1e6, 2.0)])
def test_search_report_mode_matches_oracle_ranking(cuda, fresh, num_hits, evalue, k):
    """Device ranking, -H cut and E-value cut (report mode) against the
    oracle's output_top_hits selection; k = 2 puts low scores below the
    bitscore-0 gapless hits, so those interleave with aligned hits."""
    db, qs = fresh
    ix = native.Index(db)
    r = ix.search(qs, BLOSUM62, num_hits=num_hits, report={"max_evalue": evalue, "k": k})
    opts = oracle.Opts(num_hits, evalue, 11, 1, 0.267, k, 0.14, 5, 300000, 5000)
    nsel = 0
    for q, qi in enumerate(qs):
        _, hits, _, _, nh = oracle.oracle_query(db, qi, BLOSUM62, opts)
        assert nh >= 0
        sel = oracle.oracle_rank_select(hits, num_hits, evalue)
        a, b = r["hit_off"][q], r["hit_off"][q + 1]
        assert b - a == len(sel)
        nsel += len(sel)
        assert list(r["protein"][a:b]) == [hits[i].db_index for i in sel]
        assert list(r["bitscore"][a:b]) == [hits[i].bitscore for i in sel]
        assert list(r["evalue"][a:b]) == [hits[i].evalue for i in sel]
        sw = r["sw_status"][a:b] == native.TPZ_SW_OK
        assert list(r["rawscore"][a:b][sw]) == [hits[i].rawscore for i, s in zip(sel, sw) if s]
        assert list(r["qend"][a:b][sw]) == [hits[i].qend for i, s in zip(sel, sw) if s]
        assert list(r["send"][a:b][sw]) == [hits[i].send for i, s in zip(sel, sw) if s]
    assert nsel > 0


def test_sa_search_and_hsp_stage_entry_points(cuda, fresh):
    db, qs = fresh
    ix = native.Index(db)
    orc = oracle.liboracle()
    rng = np.random.default_rng(5)
    pats = [q[i:] for q in qs[:6] for i in range(0, len(q) - 1, 7)]
    pats += [bytes(rng.integers(65, 90, L).astype(np.uint8)) for L in (1, 2, 3, 4, 5, 6, 9)]
    pats += [b"Y" * 40, b"A", b"YYYYYYYYYYYYYYYYYYYYY"]
    got = ix.sa_search(pats)
    for p, x in zip(pats, got):
        assert x == orc.orc_lower_bound(oracle._p(db.T), len(db.T), oracle._p(db.SA), p, len(p))
    # sa_hsp on random rows for every query offset kind
    qof, off, row = [], [], []
    for qi, q in enumerate(qs[:8]):
        for i in range(0, len(q), 5):
            qof.append(qi); off.append(i); row.append(int(rng.integers(0, db.Tsize)))
    sc, ln = ix.sa_hsp(qs[:8], qof, off, row, BLOSUM62)
    import ctypes
    for k in range(len(row)):
        s2, l2 = ctypes.c_int32(0), ctypes.c_int32(0)
        q = qs[qof[k]]
        orc.orc_hsp(oracle._p(db.T), ctypes.c_int64(db.Tsize), oracle._p(db.SA), q, len(q),
                    off[k], ctypes.c_int64(row[k]), oracle._p(BLOSUM62), ctypes.byref(s2), ctypes.byref(l2))
        assert ln[k] == l2.value
        if l2.value >= 0:
            assert sc[k] == s2.value


def test_search_edge_queries(cuda, fresh):
    db, qs = fresh
    ix = native.Index(db)
    plen = np.diff(db.pstart)
    pid = int(np.flatnonzero((plen > 100) & (plen < 1000))[0])
    edge = [b"", b"A", b"ACDEF", b"ACDEFG", b"V" * 50, qs[0][:6], b"Y" * 30,
            db.T[db.pstart[pid]:db.pstart[pid + 1] - 1].tobytes()]   # a DB protein itself
    r = ix.search(edge, BLOSUM62, trace_pops=1 << 14)
    opts = oracle.Opts(100, 1e-3, 11, 1, 0.267, 0.041, 0.14, 5, 300000, 5000)
    for q, qi in enumerate(edge):
        P, hits, npops, ncnt, nh = oracle.oracle_query(db, qi, BLOSUM62, opts)
        assert (r["npops"][q], r["ncounted"][q], r["hit_off"][q + 1] - r["hit_off"][q]) == (npops, ncnt, nh)
    assert r["hit_off"][1] == 0 and r["npops"][4] == 0          # empty / all-X queries
    a, b = r["hit_off"][7], r["hit_off"][8]
    top = np.argmax(r["rawscore"][a:b])
    assert r["protein"][a + top] == pid                         # finds itself


def test_index_rejects_inconsistent_files(cuda, fresh):
    db, _ = fresh
    bad = db.ind.copy()
    bad["protein_len"][3] += 1
    with pytest.raises(native.TopazError):
        native.Index(dbformat.Database(db.T, db.SA, bad, db.headers))
    sa = db.SA.copy()
    sa[10] = db.Tsize + 5
    with pytest.raises(native.TopazError):
        native.Index(dbformat.Database(db.T, sa, db.ind, db.headers))


def test_search_concurrent_calls_match_sequential(cuda, fresh):
    """tpz_search_batch from several host threads at once (each thread on its
    own default stream) gives each caller what it gets alone."""
    import threading
    db, qs = fresh
    ix = native.Index(db)
    parts = [qs[i::3] for i in range(3)]
    rep = {"max_evalue": 10.0}
    alone = [ix.search(p, BLOSUM62, report=rep) for p in parts]
    got = [None] * len(parts)

    def run(i):
        for _ in range(2):
            got[i] = ix.search(parts[i], BLOSUM62, report=rep)

    th = [threading.Thread(target=run, args=(i,)) for i in range(len(parts))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for a, b in zip(alone, got):
        for k in ("hit_off", "protein", "rawscore", "qend", "send", "bitscore", "evalue", "npops"):
            assert np.array_equal(a[k], b[k]), k


def test_index_rejects_bad_text_and_sa(cuda):
    # both checks run on the device before any kernel reads T[SA[r]] or
    # indexes the prefix table by a text byte
    db = make_db(synth.protein_db(60, seed=51))
    bad_t = dbformat.Database(db.T.copy(), db.SA, db.ind, db.headers)
    bad_t.T[3] = ord("a")
    with pytest.raises(native.TopazError, match="internal alphabet"):
        native.Index(bad_t)
    bad_sa = dbformat.Database(db.T, db.SA.copy(), db.ind, db.headers)
    bad_sa.SA[7] = db.Tsize
    with pytest.raises(native.TopazError, match="SA entry"):
        native.Index(bad_sa)
    native.Index(db).close()          # the untouched database still loads


def test_index_upload_in_pieces_matches_oracle(cuda):
    # a text whose SA (8 bytes a row) is over 64 MB goes to the device in
    # pinned pieces; searches on it match the oracle
    prot = synth.protein_db(30000, seed=61)
    db = dbformat.build_from_records([(p.encode(), s) for p, s in zip(prot.ids, prot.seqs)])
    db.SA = native.sa_build(db.T)
    assert 8 * db.Tsize > 64 << 20
    qs = [ab.aa_to_internal(s).tobytes() for s in synth.search_queries(prot, 3, 1, seed=62).seqs]
    ix = native.Index(db)
    try:
        r = ix.search(qs, BLOSUM62)
    finally:
        ix.close()
    opts = oracle.Opts(100, 1e-3, 11, 1, 0.267, 0.041, 0.14, 5, 300000, 5000)
    for q, qi in enumerate(qs):
        _, hits, npops, ncnt, nh = oracle.oracle_query(db, qi, BLOSUM62, opts)
        a, b = int(r["hit_off"][q]), int(r["hit_off"][q + 1])
        assert (r["npops"][q], r["ncounted"][q], b - a) == (npops, ncnt, nh)
        assert [int(p) for p in r["protein"][a:b]] == [h.db_index for h in hits]
