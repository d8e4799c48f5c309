"""The relink of the reference's per-hit code: its own src/ssw_wrapper.c,
compiled UNCHANGED against include/topaz_b200_ssw.h (oracle/relink/ssw.h
stands in for SSW's header) and linked against libtopaz_b200 in place of
src/ssw.c (`make -C oracle relink` -> oracle/_ref/librelink.so).  Its
get_ssw_profile + align_using_ssw_profile + stats_using_ssw_profile, driven
pair by pair as query.c drives them, must give the reference's hit fields:
the golden ssw_align scores and ends, the Karlin-Altschul doubles, and the
reference's ssw_align_stats columns."""
import ctypes
import os

import numpy as np
import pytest

import oracle
from topaz_b200 import alphabet as ab, native

pytestmark = pytest.mark.gpu
RELINK = os.path.join(os.path.dirname(oracle.REF_SO), "librelink.so")
DB_SIZE, DB_PROTEINS = 350_000_000, 1_000_000


def _idx_to_internal():
    m = np.zeros(25, np.uint8)
    for j, aa in enumerate(ab.INTERNAL_TO_AA):
        m[ab.MATRIX_ORDER.index(aa)] = ord("A") + j
    return m


def _relink():
    L = ctypes.CDLL(RELINK)
    vp = ctypes.c_void_p
    L.relink_align.argtypes = [ctypes.c_int64, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int,
                               ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                               ctypes.c_uint64, ctypes.c_uint64, vp, ctypes.c_int, vp, vp]
    return L


def _run(L, q, qoff, qlen, s, soff, slen, mat, go, ge, gapless, with_stats):
    n = len(qlen)
    oi = np.zeros((n, 8), np.int32)
    od = np.zeros((n, 3), np.float64)
    arrs = [np.ascontiguousarray(a) for a in (q, qoff.astype(np.int64), qlen.astype(np.int32), s,
                                              soff.astype(np.int64), slen.astype(np.int32))]
    L.relink_align(n, *[a.ctypes.data for a in arrs], np.ascontiguousarray(mat, np.int8).ctypes.data,
                   go, ge, 0.267, 0.041, 0.14, DB_SIZE, DB_PROTEINS,
                   np.ascontiguousarray(gapless, np.int32).ctypes.data, with_stats,
                   oi.ctypes.data, od.ctypes.data)
    return oi, od


@pytest.mark.skipif(not os.path.exists(RELINK), reason="relinked reference wrapper not built")
@pytest.mark.parametrize("key", ["BLOSUM62_11_1", "BLOSUM45_13_3"])
def test_unmodified_ssw_wrapper_relinked_gives_reference_hits(cuda, golden_sw, key):
    g = golden_sw
    L = _relink()
    name, go, ge = key.split("_")
    go, ge = int(go), int(ge)
    mat = g["mat_" + name]
    sel = np.arange(0, len(g["qlen"]), 3)
    sel = sel[g["qlen"][sel] <= 1500]
    x = _idx_to_internal()
    q, s = x[g["q"]], x[g["s"]]
    gapless = np.full(len(sel), 40, np.int32)
    gapless[::11] = 39                               # below 40: no SW (ssw_wrapper.c:171-176)
    oi, od = _run(L, q, g["qoff"][sel], g["qlen"][sel], s, g["soff"][sel], g["slen"][sel], mat,
                  go, ge, gapless, 0)
    want = g[key][:, sel]
    for j, i in enumerate(sel):
        if gapless[j] < 40:
            assert (od[j, 0], od[j, 1], oi[j, 0]) == (0.0, 1000.0, 0)
            continue
        if want[3, j] == native.TPZ_SW_DROPPED:
            assert oi[j, 0] == 32767
            continue
        assert (oi[j, 0], oi[j, 1], oi[j, 2]) == (want[0, j], want[2, j], want[1, j]), (key, i)
        assert (od[j, 0], od[j, 1]) == native.karlin(g["qlen"][i], DB_SIZE, DB_PROTEINS, oi[j, 0])


@pytest.mark.skipif(not os.path.exists(RELINK) or oracle.libref() is None,
                    reason="relinked wrapper or reference build not present")
def test_relinked_stats_match_reference_ssw_align_stats(cuda, golden_sw):
    g = golden_sw
    L, R = _relink(), oracle.libref()
    mat = g["mat_BLOSUM62"]
    want = g["BLOSUM62_11_1"]
    sel = np.flatnonzero((want[3] == 0) & (want[0] >= 30) & (g["qlen"] <= 1500))[:200]
    x = _idx_to_internal()
    oi, od = _run(L, x[g["q"]], g["qoff"][sel], g["qlen"][sel], x[g["s"]], g["soff"][sel],
                  g["slen"][sel], mat, 11, 1, np.full(len(sel), 60, np.int32), 1)
    assert len(sel) > 50
    for j, i in enumerate(sel):
        qa = np.ascontiguousarray(g["q"][g["qoff"][i]:g["qoff"][i] + g["qlen"][i]], np.int8)
        sa = np.ascontiguousarray(g["s"][g["soff"][i]:g["soff"][i] + g["slen"][i]], np.int8)
        ref = [ctypes.c_int32() for _ in range(5)] + [ctypes.c_double()]
        R.ref_ssw_stats(oracle._p(qa), ctypes.c_int32(len(qa)), oracle._p(sa), ctypes.c_int32(len(sa)),
                        oracle._p(mat), 11, 1, ctypes.c_int32(int(want[2, i])),
                        ctypes.c_int32(int(want[1, i])), ctypes.c_int32(int(want[0, i])),
                        *[ctypes.byref(v) for v in ref])
        qstart, sstart, length, gapopen, mismatch = (v.value for v in ref[:5])
        assert (oi[j, 3], oi[j, 4], oi[j, 5], oi[j, 7], oi[j, 6]) == \
            (qstart, sstart, length, gapopen, mismatch), i
        assert od[j, 2] == ref[5].value
