"""The per-call seam shims tpz_sa_search and tpz_sa_hsp (the argument lists
of src/search.h:13-14 over the resident index) against the reference's own
sa_search and sa_hsp run on the same database (oracle/_ref stage drivers):
every output of every call, including sa_search's match count and last
compared prefix length, over whole query suffixes (as query.c:110 calls it),
fixed-length patterns, patterns that end the text, and the empty-pattern
error."""
import ctypes

import numpy as np
import pytest

import oracle
from topaz_b200 import alphabet as ab, dbformat, native, synth

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(oracle.libref() is None, reason="reference build not present")]


@pytest.fixture(scope="module")
def both(cuda):
    R = oracle.libref()
    prot = synth.protein_db(2500, seed=311)
    db = dbformat.build_from_records([(p.encode(), s) for p, s in zip(prot.ids, prot.seqs)])
    SA = np.zeros(db.Tsize, np.int64)
    assert R.divsufsort64(oracle._p(db.T), oracle._p(SA), ctypes.c_int64(db.Tsize)) == 0
    db.SA = SA
    h = R.ref_db_open(oracle._p(db.T), ctypes.c_uint64(db.Tsize), oracle._p(SA), oracle._p(db.ind),
                      ctypes.c_uint64(db.Psize), db.headers, ctypes.c_uint64(len(db.headers)))
    ix = native.Index(db)
    L = native.lib()
    i64p = ctypes.POINTER(ctypes.c_int64)
    L.tpz_sa_search.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int64,
                                ctypes.c_int64, i64p, i64p, i64p]
    i32p = ctypes.POINTER(ctypes.c_int32)
    L.tpz_sa_hsp.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32,
                             ctypes.c_int64, ctypes.c_void_p, i32p, i32p]
    qs = [ab.aa_to_internal(s).tobytes() for s in synth.search_queries(prot, 6, 3, seed=312).seqs]
    yield R, h, L, ix, db, prot, qs
    ix.close()
    R.ref_db_close(ctypes.c_void_p(h))


def _search(R, h, L, ix, q, off, length):
    want = [ctypes.c_int64() for _ in range(3)]
    rw = R.ref_sa_search(ctypes.c_void_p(h), q, len(q), ctypes.c_int64(off), ctypes.c_int64(length),
                         *[ctypes.byref(x) for x in want])
    got = [ctypes.c_int64() for _ in range(3)]
    rg = L.tpz_sa_search(ix.handle, q, len(q), off, length, *[ctypes.byref(x) for x in got])
    return (rw, [x.value for x in want]), (rg, [x.value for x in got])


def test_sa_search_shim_every_output_matches_reference(both):
    R, h, L, ix, db, prot, qs = both
    n = 0
    for q in qs:
        for off in range(0, len(q) - 5, 3):
            for length in (0, 1, 3, 6, 12):
                if off + length > len(q):
                    continue                   # sa_search would read past the query
                w, g = _search(R, h, L, ix, q, off, length)
                assert w == g, (off, length)
                n += 1
    # patterns copied from the text: matches exist, some run to a protein end
    T = db.T.tobytes()
    rng = np.random.default_rng(5)
    for start in rng.integers(0, db.Tsize - 40, 150):
        p = T[start:start + 30].split(b"\n")[0]
        if len(p) < 2:
            continue
        w, g = _search(R, h, L, ix, p, 0, 0)
        assert w == g and g[1][1] >= 1
        n += 1
    assert n > 1500


def test_sa_search_shim_empty_pattern_is_an_error(both):
    R, h, L, ix, db, prot, qs = both
    q = qs[0]
    w, g = _search(R, h, L, ix, q, len(q), 0)
    assert w[0] == g[0] == -1 and w[1][0] == g[1][0] == -1


def test_sa_hsp_shim_matches_reference(both):
    R, h, L, ix, db, prot, qs = both
    mat = np.ascontiguousarray(synth.matrix("BLOSUM62"), np.int8)
    rng = np.random.default_rng(6)
    for q in qs[:5]:
        for off in range(0, len(q), 7):
            pos = ix.sa_search([q[off:]])[0]
            for row in {max(pos - 1, 0), min(pos, db.Tsize - 1), int(rng.integers(0, db.Tsize))}:
                ws, wl = ctypes.c_int32(), ctypes.c_int32()
                R.ref_hsp(ctypes.c_void_p(h), q, len(q), off, ctypes.c_int64(row), b"BLOSUM62",
                          ctypes.byref(ws), ctypes.byref(wl))
                gs, gl = ctypes.c_int32(), ctypes.c_int32()
                assert L.tpz_sa_hsp(ix.handle, q, len(q), off, row, mat.ctypes.data,
                                    ctypes.byref(gs), ctypes.byref(gl)) == 0
                assert (gs.value, gl.value) == (ws.value, wl.value), (off, row)
