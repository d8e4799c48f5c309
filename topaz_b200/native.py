"""ctypes binding of libtopaz_b200.so (the C ABI in include/topaz_b200.h).

There is no fallback: if the native library is missing or a call fails the
functions raise.  Device entry points take raw device pointers (ints) and a
stream handle; the helpers accept torch CUDA tensors.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

_LIB = None

TPZ_SW_OK, TPZ_SW_DROPPED, TPZ_SW_INVALID = 0, 1, 2

_VP = ctypes.c_void_p
_I64 = ctypes.c_int64
_I32 = ctypes.c_int


class TopazError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("topaz_b200 error %d: %s" % (code, msg))
        self.code = code


def lib_path() -> str:
    return _build.LIB


def lib():
    """Loads the native library (building it first if it is missing here)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = _build.LIB
    if not os.path.exists(path):
        _build.build()
    if not os.path.exists(path):
        raise ImportError("libtopaz_b200.so is not built (%s)" % path)
    L = ctypes.CDLL(path)
    L.tpz_last_error.restype = ctypes.c_char_p
    L.tpz_version.restype = ctypes.c_char_p
    L.tpz_matrix.argtypes = [ctypes.c_char_p, _VP]
    sw_args = [_I64, _VP, _VP, _VP, _VP, _VP, _VP, _VP, _I32, _I32, _VP, _VP, _VP, _VP]
    L.tpz_sw_batch_host.argtypes = sw_args
    L.tpz_sw_batch_device.argtypes = sw_args + [_VP]
    L.tpz_sw_last_launches.restype = ctypes.c_int64
    L.tpz_sw_align_one.argtypes = [_VP, _I32, _VP, _I32, _VP, _I32, _I32, _VP, _VP]
    L.tpz_dpx_probe.argtypes = [_I64, _I32, _VP, _VP, _VP]
    _LIB = L
    return L


def check(rc: int):
    if rc != 0:
        raise TopazError(rc, lib().tpz_last_error().decode(errors="replace"))


def _p(a: np.ndarray):
    return a.ctypes.data_as(_VP)


def matrix(name: str = "BLOSUM62") -> np.ndarray:
    out = np.zeros(625, dtype=np.int8)
    check(lib().tpz_matrix(name.encode(), _p(out)))
    return out.reshape(25, 25)


def sw_batch_host(q, qoff, qlen, s, soff, slen, mat, gap_open=11, gap_extend=1):
    """Host buffers in, host results out (score, ref_end, read_end, status)."""
    n = len(qlen)
    q = np.ascontiguousarray(q, dtype=np.int8)
    s = np.ascontiguousarray(s, dtype=np.int8)
    qoff = np.ascontiguousarray(qoff, dtype=np.int64)
    soff = np.ascontiguousarray(soff, dtype=np.int64)
    qlen = np.ascontiguousarray(qlen, dtype=np.int32)
    slen = np.ascontiguousarray(slen, dtype=np.int32)
    mat = np.ascontiguousarray(mat, dtype=np.int8)
    out = [np.zeros(n, dtype=np.int32) for _ in range(4)]
    check(lib().tpz_sw_batch_host(n, _p(q), _p(qoff), _p(qlen), _p(s), _p(soff), _p(slen),
                                  _p(mat), gap_open, gap_extend, *[_p(o) for o in out]))
    return tuple(out)


def sw_batch_device(n, q_ptr, qoff_ptr, qlen_ptr, s_ptr, soff_ptr, slen_ptr, mat, gap_open,
                    gap_extend, score_ptr, ref_end_ptr, read_end_ptr, status_ptr, stream=0):
    """Device pointers in and out; enqueues on `stream` (cudaStream_t as int)."""
    mat = np.ascontiguousarray(mat, dtype=np.int8)
    check(lib().tpz_sw_batch_device(n, q_ptr, qoff_ptr, qlen_ptr, s_ptr, soff_ptr, slen_ptr,
                                    _p(mat), gap_open, gap_extend, score_ptr, ref_end_ptr,
                                    read_end_ptr, status_ptr, stream))


def sw_batch_torch(t, mat, gap_open=11, gap_extend=1, stream=None):
    """`t`: dict of CUDA tensors q, qoff, qlen, s, soff, slen, score, ref_end,
    read_end, status.  Enqueues on `stream` (torch.cuda.Stream) or the
    current stream."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    sw_batch_device(int(t["qlen"].numel()), t["q"].data_ptr(), t["qoff"].data_ptr(),
                    t["qlen"].data_ptr(), t["s"].data_ptr(), t["soff"].data_ptr(),
                    t["slen"].data_ptr(), mat, gap_open, gap_extend, t["score"].data_ptr(),
                    t["ref_end"].data_ptr(), t["read_end"].data_ptr(), t["status"].data_ptr(),
                    st.cuda_stream)


def sw_align_one(q_ptr, qlen, s_ptr, slen, mat, gap_open, gap_extend, out4_ptr, stream=0):
    """One pair, one kernel launch (tpz_sw_align_one): device pointers to the
    query and subject (matrix indices) and to 4 int32 outputs {score,
    ref_end, read_end, status}; enqueued on `stream` (a cudaStream_t)."""
    L = lib()
    check(L.tpz_sw_align_one(q_ptr, int(qlen), s_ptr, int(slen), _p(np.ascontiguousarray(mat, np.int8)),
                             gap_open, gap_extend, out4_ptr, stream))


def sa_build(T) -> np.ndarray:
    """Suffix array of the text T (uint8) built on the device (tpz_sa_build)."""
    L = lib()
    L.tpz_sa_build.argtypes = [_VP, _I64, _VP, _VP]
    T = np.ascontiguousarray(T, dtype=np.uint8)
    SA = np.empty(max(len(T), 1), np.int64)
    check(L.tpz_sa_build(_p(T), len(T), _p(SA), None))
    return SA[:len(T)]


def last_launches() -> int:
    return int(lib().tpz_sw_last_launches())


def dpx_probe(blocks, iters, out_ptr, stream=0) -> int:
    """Enqueues the DPX throughput probe; returns the number of DPX ops."""
    ops = ctypes.c_int64()
    check(lib().tpz_dpx_probe(blocks, iters, out_ptr, stream, ctypes.byref(ops)))
    return ops.value


# ------------------------------------------------------------------ search

class _SearchOpts(ctypes.Structure):
    _fields_ = [("num_hits", ctypes.c_int32), ("gap_open", ctypes.c_int32),
                ("gap_extend", ctypes.c_int32), ("min_hit_length", ctypes.c_int32),
                ("seeds", ctypes.c_int32), ("alignments", ctypes.c_int32),
                ("mat625", _VP), ("trace_pops", ctypes.c_int64),
                ("report_hits", ctypes.c_int32), ("max_evalue", ctypes.c_double),
                ("lam", ctypes.c_double), ("k", ctypes.c_double), ("H", ctypes.c_double),
                ("db_size", ctypes.c_uint64), ("db_proteins", ctypes.c_uint64),
                ("blasttab_stats", ctypes.c_int32), ("ingest", ctypes.c_int32)]


_P64 = ctypes.POINTER(ctypes.c_int64)
_P32 = ctypes.POINTER(ctypes.c_int32)


class _SearchResult(ctypes.Structure):
    _fields_ = [("nq", ctypes.c_int64), ("nhits_total", ctypes.c_int64),
                ("hit_off", _P64), ("npops", _P64), ("ncounted", _P64), ("status", _P32),
                ("protein", _P32), ("gapless_score", _P32), ("gapless_length", _P32),
                ("suffix_offset", _P32), ("rawscore", _P32), ("qend", _P32), ("send", _P32),
                ("sw_status", _P32), ("trace_n", _P64), ("trace_row", _P64),
                ("trace_off", _P32), ("trace_score", _P32), ("trace_len", _P32),
                ("trace_counted", _P32), ("stage_ms", ctypes.c_double * 4),
                ("bitscore", ctypes.POINTER(ctypes.c_double)),
                ("evalue", ctypes.POINTER(ctypes.c_double)),
                ("sw_pairs", ctypes.c_int64), ("sw_cells", ctypes.c_int64),
                ("seed_ms", ctypes.c_double), ("chain_ms", ctypes.c_double),
                ("positions", ctypes.c_int64), ("qstart", _P32), ("sstart", _P32),
                ("length", _P32), ("gapopen", _P32), ("mismatch", _P32),
                ("identity", ctypes.POINTER(ctypes.c_double)),
                ("chain_elems", ctypes.c_int64), ("refill_elems", ctypes.c_int64)]


def _search_sigs(L):
    if getattr(L, "_search_sigs", False):
        return
    L.tpz_index_create.argtypes = [_VP, _I64, _VP, _VP, _I64, ctypes.POINTER(_VP)]
    L.tpz_index_destroy.argtypes = [_VP]
    L.tpz_index_device_bytes.argtypes = [_VP]
    L.tpz_index_device_bytes.restype = ctypes.c_int64
    L.tpz_sa_search_batch.argtypes = [_VP, _VP, _VP, _VP, _I64, _VP]
    L.tpz_sa_hsp_batch.argtypes = [_VP, _VP, _VP, _VP, _I64, _VP, _VP, _VP, _I64, _VP, _VP, _VP]
    L.tpz_search_batch.argtypes = [_VP, _VP, _VP, _VP, _I64, ctypes.POINTER(_SearchOpts),
                                   ctypes.POINTER(ctypes.POINTER(_SearchResult))]
    L.tpz_search_result_free.argtypes = [ctypes.POINTER(_SearchResult)]
    L.tpz_karlin.argtypes = [ctypes.c_int32, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                             ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    L.tpz_search_query_device_bytes.argtypes = [ctypes.c_int32, ctypes.POINTER(_SearchOpts)]
    L.tpz_search_query_device_bytes.restype = ctypes.c_int64
    L._search_sigs = True


def _concat(seqs):
    """list of bytes -> (cat uint8, off int64, len int32)"""
    lens = np.array([len(s) for s in seqs], dtype=np.int32)
    off = np.zeros(len(seqs), dtype=np.int64)
    if len(seqs) > 1:
        off[1:] = np.cumsum(lens, dtype=np.int64)[:-1]
    cat = np.frombuffer(b"".join(seqs) + b"\0", dtype=np.uint8)
    return cat, off, lens


class Index:
    """A database resident in device memory (tpz_index)."""

    def __init__(self, db):
        L = lib()
        _search_sigs(L)
        self.db = db
        self._T = np.ascontiguousarray(db.T, dtype=np.uint8)
        self._SA = np.ascontiguousarray(db.SA, dtype=np.int64)
        self._ind = np.ascontiguousarray(db.ind)
        h = _VP()
        check(L.tpz_index_create(_p(self._T), len(self._T), _p(self._SA), _p(self._ind),
                                 len(self._ind), ctypes.byref(h)))
        self.handle = h

    def close(self):
        if self.handle:
            lib().tpz_index_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self):
        return int(lib().tpz_index_device_bytes(self.handle))

    def sa_search(self, patterns):
        cat, off, lens = _concat(patterns)
        out = np.zeros(len(patterns), dtype=np.int64)
        check(lib().tpz_sa_search_batch(self.handle, _p(cat), _p(off), _p(lens), len(patterns),
                                        _p(out)))
        return out

    def sa_hsp(self, queries, query_of, qoffset, row, mat):
        cat, off, lens = _concat(queries)
        query_of = np.ascontiguousarray(query_of, dtype=np.int32)
        qoffset = np.ascontiguousarray(qoffset, dtype=np.int32)
        row = np.ascontiguousarray(row, dtype=np.int64)
        mat = np.ascontiguousarray(mat, dtype=np.int8)
        n = len(row)
        sc = np.zeros(n, dtype=np.int32)
        ln = np.zeros(n, dtype=np.int32)
        check(lib().tpz_sa_hsp_batch(self.handle, _p(cat), _p(off), _p(lens), len(queries),
                                     _p(query_of), _p(qoffset), _p(row), n, _p(mat), _p(sc),
                                     _p(ln)))
        return sc, ln

    def search(self, queries, mat, num_hits=100, gap_open=11, gap_extend=1, min_hit_length=5,
               seeds=300000, alignments=5000, trace_pops=0, report=None, ingest=0):
        """Runs a batch of queries (internal-alphabet bytes).  Returns a dict
        of numpy arrays (per query: hit_off, npops, ncounted, status; per hit:
        protein, gapless_score, gapless_length, suffix_offset, rawscore,
        qend, send, sw_status; optional trace_*).

        report: None for every hit in traversal order, or a dict with
        max_evalue (and optionally hits, lam, k, H, db_size, db_proteins,
        stats) for the ranked, E-value-cut top hits with bitscore and evalue
        arrays; with stats=True also the --blasttab columns (qstart, sstart,
        length, gapopen, mismatch, identity) computed on the device."""
        L = lib()
        cat, off, lens = _concat(queries)
        mat = np.ascontiguousarray(mat, dtype=np.int8)
        o = _SearchOpts(num_hits, gap_open, gap_extend, min_hit_length, seeds, alignments,
                        _p(mat), trace_pops)
        o.ingest = int(ingest)
        if report is not None:
            T, P = len(self._T), len(self._ind)
            o.report_hits = int(report.get("hits", num_hits))
            o.max_evalue = float(report.get("max_evalue", 1e-3))
            o.lam = float(report.get("lam", 0.267))
            o.k = float(report.get("k", 0.041))
            o.H = float(report.get("H", 0.140))
            o.db_size = int(report.get("db_size", T - P))
            o.db_proteins = int(report.get("db_proteins", P))
            o.blasttab_stats = 1 if report.get("stats") else 0
        res = ctypes.POINTER(_SearchResult)()
        check(L.tpz_search_batch(self.handle, _p(cat), _p(off), _p(lens), len(queries),
                                 ctypes.byref(o), ctypes.byref(res)))
        try:
            r = res.contents
            nq, nh = r.nq, r.nhits_total

            def arr(ptr, n):
                return np.ctypeslib.as_array(ptr, shape=(n,)).copy() if n else np.zeros(0, np.int64)

            out = {"hit_off": arr(r.hit_off, nq + 1), "npops": arr(r.npops, nq),
                   "ncounted": arr(r.ncounted, nq), "status": arr(r.status, nq)}
            for k in ("protein", "gapless_score", "gapless_length", "suffix_offset", "rawscore",
                      "qend", "send", "sw_status"):
                out[k] = arr(getattr(r, k), nh)
            out["stage_ms"] = list(r.stage_ms)
            out["sw_pairs"], out["sw_cells"] = int(r.sw_pairs), int(r.sw_cells)
            out["seed_ms"], out["chain_ms"] = float(r.seed_ms), float(r.chain_ms)
            out["positions"] = int(r.positions)
            out["chain_elems"], out["refill_elems"] = int(r.chain_elems), int(r.refill_elems)
            if report is not None:
                out["bitscore"] = arr(r.bitscore, nh)
                out["evalue"] = arr(r.evalue, nh)
                if report.get("stats"):
                    for k in ("qstart", "sstart", "length", "gapopen", "mismatch", "identity"):
                        out[k] = arr(getattr(r, k), nh)
            if trace_pops:
                out["trace_n"] = arr(r.trace_n, nq)
                for k in ("trace_row", "trace_off", "trace_score", "trace_len", "trace_counted"):
                    out[k] = arr(getattr(r, k), nq * trace_pops).reshape(nq, trace_pops)
            return out
        finally:
            L.tpz_search_result_free(res)


def query_device_bytes(qlen, num_hits=100, alignments=5000, min_hit_length=5,
                       seeds=300000, gap_open=11, gap_extend=1):
    """tpz_search_query_device_bytes: device memory of one query in a batch."""
    L = lib()
    _search_sigs(L)
    o = _SearchOpts(num_hits, gap_open, gap_extend, min_hit_length, seeds, alignments, None, 0)
    v = L.tpz_search_query_device_bytes(int(qlen), ctypes.byref(o))
    if v < 0:
        raise TopazError(-1, "bad arguments")
    return int(v)


def karlin(qlen, db_size, db_proteins, raw, lam=0.267, k=0.041, H=0.14):
    """(bitscore, evalue) as align_using_ssw_profile computes them."""
    L = lib()
    _search_sigs(L)
    b, e = ctypes.c_double(), ctypes.c_double()
    L.tpz_karlin(int(qlen), int(db_size), int(db_proteins), lam, k, H, int(raw),
                 ctypes.byref(b), ctypes.byref(e))
    return b.value, e.value


def seg_mask(residues: bytes) -> bytes:
    """SEG hard-masking of upper-cased residues (tpzh_seg_mask)."""
    L = lib()
    L.tpzh_seg_mask.argtypes = [ctypes.c_char_p, ctypes.c_int]
    buf = ctypes.create_string_buffer(residues, len(residues))
    L.tpzh_seg_mask(buf, len(residues))
    return buf.raw[:len(residues)]


def prepare_queries(queries, seg: bool = True, threads: int = 0):
    """prepare_query for a list of queries in one library call
    (tpz_prepare_queries), on `threads` host threads (0: all cores)."""
    L = lib()
    L.tpz_prepare_queries.argtypes = [_VP, _VP, _VP, _I64, ctypes.c_int, ctypes.c_int]
    cat, off, lens = _concat(queries)
    cat = cat.copy()
    check(L.tpz_prepare_queries(_p(cat), _p(off), _p(lens), len(queries), 1 if seg else 0,
                                threads or (os.cpu_count() or 1)))
    b = cat.tobytes()
    return [b[o:o + n] for o, n in zip(off.tolist(), lens.tolist())]


def prepare_query(residues: bytes, seg: bool = True) -> bytes:
    """A FASTA query as the search kernels take it: SEG (unless disabled),
    then the internal alphabet (run_seg + seq_2internal)."""
    from . import alphabet as ab
    if seg:
        residues = seg_mask(residues)
    return ab.aa_to_internal(np.frombuffer(residues, np.uint8)).tobytes()
