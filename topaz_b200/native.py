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


def last_launches() -> int:
    return int(lib().tpz_sw_last_launches())


def dpx_probe(blocks, iters, out_ptr, stream=0) -> int:
    """Enqueues the DPX throughput probe; returns the number of DPX ops."""
    ops = ctypes.c_int64()
    check(lib().tpz_dpx_probe(blocks, iters, out_ptr, stream, ctypes.byref(ops)))
    return ops.value
