"""The SSW-named per-call shims (include/topaz_b200_ssw.h) give the
reference's ssw_align and ssw_align_stats results pair by pair."""
import ctypes

import numpy as np
import pytest

import oracle
from topaz_b200 import native, synth

pytestmark = pytest.mark.gpu


class SAlign(ctypes.Structure):
    _fields_ = [("score1", ctypes.c_uint16), ("score2", ctypes.c_uint16),
                ("ref_begin1", ctypes.c_int32), ("ref_end1", ctypes.c_int32),
                ("read_begin1", ctypes.c_int32), ("read_end1", ctypes.c_int32),
                ("ref_end2", ctypes.c_int32), ("cigar", ctypes.c_void_p), ("cigarLen", ctypes.c_int32)]


def _lib():
    L = native.lib()
    L.ssw_init.restype = ctypes.c_void_p
    L.ssw_init.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int8]
    L.init_destroy.argtypes = [ctypes.c_void_p]
    L.ssw_align.restype = ctypes.POINTER(SAlign)
    L.ssw_align.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint8,
                            ctypes.c_uint8, ctypes.c_uint8, ctypes.c_uint16, ctypes.c_int32,
                            ctypes.c_int32]
    L.align_destroy.argtypes = [ctypes.POINTER(SAlign)]
    o = ctypes.POINTER(ctypes.c_int32)
    L.ssw_align_stats.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint8,
                                  ctypes.c_uint8, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                  ctypes.c_uint16, o, o, o, o, o, ctypes.POINTER(ctypes.c_double)]
    return L


def _align(L, q, s, mat, go, ge):
    prof = L.ssw_init(q.ctypes.data, len(q), mat.ctypes.data, 25, 2)
    assert prof
    try:
        r = L.ssw_align(prof, s.ctypes.data, len(s), go, ge, 0, 0, 0, 15)
        if not r:
            return None
        a = r.contents
        out = (a.score1, a.ref_end1, a.read_end1, a.ref_begin1, a.read_begin1, a.score2, a.cigarLen)
        L.align_destroy(r)
        return out
    finally:
        L.init_destroy(prof)


def test_ssw_align_shim_matches_reference_golden(cuda, golden_sw):
    g = golden_sw
    L = _lib()
    for key in ("BLOSUM62_11_1", "BLOSUM45_13_3", "PAM30_9_1"):
        name, go, ge = key.split("_")
        mat = np.ascontiguousarray(g["mat_" + name], np.int8)
        want = g[key]
        for i in range(0, len(g["qlen"]), 7):
            q = np.ascontiguousarray(g["q"][g["qoff"][i]:g["qoff"][i] + g["qlen"][i]], np.int8)
            s = np.ascontiguousarray(g["s"][g["soff"][i]:g["soff"][i] + g["slen"][i]], np.int8)
            got = _align(L, q, s, mat, int(go), int(ge))
            if want[3, i] == native.TPZ_SW_DROPPED:
                assert got is None, i
            else:
                assert got[:3] == tuple(int(x) for x in want[:3, i]), (key, i)
                assert got[3:] == (-1, -1, 0, 0)


def test_ssw_align_shim_long_queries(cuda):
    """Queries past 1024 residues take the batched kernels inside ssw_align."""
    L = _lib()
    ps = synth.sw_pairs(24, seed=81, homolog_frac=0.5, q_range=(1100, 2600), s_range=(200, 3000))
    mat = synth.matrix("BLOSUM62")
    sc, re_, rd, st = oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, 11, 1)
    for i in range(ps.n):
        q = np.ascontiguousarray(ps.q[ps.qoff[i]:ps.qoff[i] + ps.qlen[i]], np.int8)
        s = np.ascontiguousarray(ps.s[ps.soff[i]:ps.soff[i] + ps.slen[i]], np.int8)
        got = _align(L, q, s, mat, 11, 1)
        assert got is not None and got[:3] == (sc[i], re_[i], rd[i]), i


@pytest.mark.skipif(oracle.libref() is None, reason="reference build not present")
def test_ssw_align_stats_shim_matches_reference(cuda):
    L, R = _lib(), oracle.libref()
    ps = synth.sw_pairs(150, seed=82, homolog_frac=0.7, q_range=(20, 900), s_range=(20, 1500))
    mat = synth.matrix("BLOSUM62")
    sc, re_, rd, st = oracle.reference_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, 11, 1)
    n = 0
    for i in range(ps.n):
        if st[i] != 0 or sc[i] < 30:
            continue
        q = np.ascontiguousarray(ps.q[ps.qoff[i]:ps.qoff[i] + ps.qlen[i]], np.int8)
        s = np.ascontiguousarray(ps.s[ps.soff[i]:ps.soff[i] + ps.slen[i]], np.int8)
        ref = [ctypes.c_int32() for _ in range(5)] + [ctypes.c_double()]
        R.ref_ssw_stats(oracle._p(q), ctypes.c_int32(len(q)), oracle._p(s), ctypes.c_int32(len(s)),
                        oracle._p(mat), 11, 1, ctypes.c_int32(rd[i]), ctypes.c_int32(re_[i]),
                        ctypes.c_int32(sc[i]), *[ctypes.byref(x) for x in ref])
        mine = [ctypes.c_int32() for _ in range(5)] + [ctypes.c_double()]
        prof = L.ssw_init(q.ctypes.data, len(q), mat.ctypes.data, 25, 2)
        L.ssw_align_stats(prof, s.ctypes.data, len(s), 11, 1, 15, int(rd[i]), int(re_[i]), int(sc[i]),
                          *[ctypes.byref(x) for x in mine])
        L.init_destroy(prof)
        assert [x.value for x in mine] == [x.value for x in ref], i
        n += 1
    assert n > 20
