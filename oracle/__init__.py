"""Python access to the oracle (test infrastructure only).

`liboracle()`  -- the CPU restatement (oracle.c), built on demand with make.
`libref()`     -- the unmodified reference compiled into _ref/ (None when it
                  was not built; it needs the TOPAZ sources to build).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
this module, and only as the checker / the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtopazref.so")
REF_BIN = os.path.join(HERE, "_ref", "topaz")
# the TOPAZ source tree (its src/ directory) to compile the reference checker
# from; unset where the sources are not present (a host that only runs the
# prebuilt _ref/)
REF_SRC = os.environ.get("TOPAZ_REF_SRC", "")

_VP = ctypes.c_void_p
_orc = None
_ref = None


def build_oracle():
    subprocess.check_call(["make", "-s", "-C", HERE, "liboracle.so"])


def build_ref():
    """Compiles the reference sources where they lie (development container
    only).  Returns False when the sources are not present."""
    if not REF_SRC or not os.path.isdir(REF_SRC):
        return False
    subprocess.check_call(["make", "-s", "-C", HERE, "-j8", "ref", "REF=" + REF_SRC])
    # the reference's ssw_wrapper.c relinked against the library (needs
    # libtopaz_b200.so built first)
    subprocess.check_call(["make", "-s", "-C", HERE, "relink", "REF=" + REF_SRC])
    return True


class OHit(ctypes.Structure):
    _fields_ = [("db_index", ctypes.c_int64)] + [
        (n, ctypes.c_int32) for n in
        "gapless_score gapless_length suffix_offset is_aligned rawscore qend send status".split()
    ] + [("bitscore", ctypes.c_double), ("evalue", ctypes.c_double)]


class RHit(ctypes.Structure):
    _fields_ = [("db_index", ctypes.c_int64)] + [
        (n, ctypes.c_int32) for n in
        ("gapless_score gapless_length suffix_offset is_aligned rawscore qstart qend sstart send "
         "length mismatch gapopen pad").split()
    ] + [(n, ctypes.c_double) for n in ("identity", "bitscore", "evalue")]


class Opts(ctypes.Structure):
    _fields_ = [("num_hits", ctypes.c_int32), ("evalue", ctypes.c_double),
                ("gap_open", ctypes.c_int32), ("gap_extend", ctypes.c_int32),
                ("lambda_", ctypes.c_double), ("k", ctypes.c_double), ("H", ctypes.c_double),
                ("min_hit_length", ctypes.c_int32), ("seeds", ctypes.c_int32),
                ("alignments", ctypes.c_int32)]


def liboracle():
    global _orc
    if _orc is None:
        src = os.path.join(HERE, "oracle.c")
        if not os.path.exists(ORACLE_SO) or os.path.getmtime(src) > os.path.getmtime(ORACLE_SO):
            build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_lower_bound.restype = ctypes.c_int64
        _orc = L
    return _orc


def libref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            return None
        L = ctypes.CDLL(REF_SO)
        L.ref_db_open.restype = _VP
        L.ref_matrix.restype = ctypes.POINTER(ctypes.c_int8)
        _ref = L
    return _ref


def _p(a):
    return a.ctypes.data_as(_VP)


def _sw_batch(L, fn, q, qoff, qlen, s, soff, slen, mat, go, ge, nthreads):
    n = len(qlen)
    q = np.ascontiguousarray(q, np.int8); s = np.ascontiguousarray(s, np.int8)
    qoff = np.ascontiguousarray(qoff, np.int64); soff = np.ascontiguousarray(soff, np.int64)
    qlen = np.ascontiguousarray(qlen, np.int32); slen = np.ascontiguousarray(slen, np.int32)
    mat = np.ascontiguousarray(mat, np.int8)
    out = [np.zeros(n, np.int32) for _ in range(4)]
    getattr(L, fn)(ctypes.c_int64(n), _p(q), _p(qoff), _p(qlen), _p(s), _p(soff), _p(slen),
                   _p(mat), ctypes.c_int(go), ctypes.c_int(ge), ctypes.c_int(nthreads),
                   *[_p(o) for o in out])
    return tuple(out)


def oracle_sw(q, qoff, qlen, s, soff, slen, mat, go=11, ge=1, nthreads=None):
    """(score, ref_end, read_end, status) from the CPU restatement."""
    return _sw_batch(liboracle(), "orc_ssw_batch", q, qoff, qlen, s, soff, slen, mat, go, ge,
                     nthreads or os.cpu_count() or 1)


def reference_sw(q, qoff, qlen, s, soff, slen, mat, go=11, ge=1, nthreads=None):
    """(score, ref_end, read_end, status) from the reference ssw_align."""
    L = libref()
    if L is None:
        raise FileNotFoundError("oracle/_ref is not built")
    return _sw_batch(L, "ref_ssw_batch", q, qoff, qlen, s, soff, slen, mat, go, ge,
                     nthreads or os.cpu_count() or 1)


def oracle_query(db, qint: bytes, mat, opts: Opts, max_pops=1 << 20, max_hits=8192):
    """Runs one query through the restatement; returns (pops, hits, npops,
    ncounted) with pops a dict of arrays and hits a list of OHit."""
    L = liboracle()
    rows = np.zeros(max_pops, np.int64)
    arr = [np.zeros(max_pops, np.int32) for _ in range(4)]
    npops, ncnt = ctypes.c_int64(), ctypes.c_int64()
    hits = (OHit * max_hits)()
    T = np.ascontiguousarray(db.T)
    SA = np.ascontiguousarray(db.SA, np.int64)
    ps = np.ascontiguousarray(db.pstart, np.int64)
    mat = np.ascontiguousarray(mat, np.int8)
    nh = L.orc_query_run(_p(T), ctypes.c_int64(len(T)), _p(SA), _p(ps), ctypes.c_int64(len(ps)),
                         qint, ctypes.c_int32(len(qint)), _p(mat), ctypes.byref(opts),
                         _p(rows), *[_p(a) for a in arr], ctypes.c_int64(max_pops),
                         ctypes.byref(npops), ctypes.byref(ncnt), hits, ctypes.c_int32(max_hits))
    n = min(npops.value, max_pops)
    pops = {"row": rows[:n], "off": arr[0][:n], "score": arr[1][:n], "len": arr[2][:n],
            "counted": arr[3][:n]}
    return pops, list(hits[:max(nh, 0)]), npops.value, ncnt.value, nh


def oracle_rank_select(hits, num_hits, evalue):
    """Indices into `hits` (traversal order) of the lines output_top_hits
    prints, in print order."""
    L = liboracle()
    arr = (OHit * max(len(hits), 1))(*hits)
    out = np.zeros(max(len(hits), 1), np.int32)
    k = L.orc_rank_select(arr, ctypes.c_int32(len(hits)), ctypes.c_int32(num_hits),
                          ctypes.c_double(evalue), _p(out))
    return [int(i) for i in out[:k]]
