"""The allocation-free batched SW entry point, tpz_sw_batch_device_noalloc.

It exists for callers that may not have device memory allocated on their
behalf (a server running against a planned HBM budget, or a loop that cannot
take the device-wide synchronization of cudaMalloc/cudaFree).  Its results
must equal those of tpz_sw_batch_device exactly, also on the second of two
calls in a row (the shared static scratch keeps the previous call's
contents).  Collected last so that a run stopping at the first failure has
run every other test before it."""
import ctypes

import numpy as np
import pytest

from topaz_b200 import native, synth

pytestmark = pytest.mark.gpu

MAX_PAIRS = 65536
_FIELDS = ("score", "ref_end", "read_end", "status")


def _device_pairs(torch, ps):
    d = torch.device("cuda:0")
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(ps, k))).to(d)
         for k in ("q", "qoff", "qlen", "s", "soff", "slen")}
    for k in _FIELDS:
        t[k] = torch.full((ps.n,), -7, dtype=torch.int32, device=d)
    return t


def _call_noalloc(torch, t, n, mat, go=11, ge=1):
    L = native.lib()
    L.tpz_sw_batch_device_noalloc.argtypes = [ctypes.c_int64] + [ctypes.c_void_p] * 7 + \
        [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 5
    for k in _FIELDS:
        t[k].fill_(-7)
    rc = L.tpz_sw_batch_device_noalloc(
        n, *[t[k].data_ptr() for k in ("q", "qoff", "qlen", "s", "soff", "slen")],
        np.ascontiguousarray(mat, np.int8).ctypes.data, go, ge,
        *[t[k].data_ptr() for k in _FIELDS], torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return rc, np.stack([t[k].cpu().numpy() for k in _FIELDS])


def test_noalloc_matches_allocating_entry_point_twice(cuda):
    torch = cuda
    ps = synth.sw_pairs(20000, seed=77, q_range=(1, 1024), s_range=(0, 3000))
    mat = synth.matrix("BLOSUM62")
    t = _device_pairs(torch, ps)
    native.sw_batch_torch(t, mat, 11, 1)
    torch.cuda.synchronize()
    ref = np.stack([t[k].cpu().numpy() for k in _FIELDS])
    assert (ref[3] == native.TPZ_SW_OK).all()
    assert (ref[0] >= 251).sum() > 100               # the i16 rerun path is exercised
    for _ in range(2):
        rc, got = _call_noalloc(torch, t, ps.n, mat)
        assert rc == 0, native.lib().tpz_last_error()
        assert (got == ref).all()


def test_noalloc_smaller_batch_after_larger(cuda):
    # a second, smaller call must not see the first call's bins or reruns
    torch = cuda
    mat = synth.matrix("BLOSUM50")
    big = synth.sw_pairs(MAX_PAIRS, seed=5, q_range=(1, 1024), s_range=(0, 1500))
    small = synth.sw_pairs(333, seed=6, q_range=(1, 1024), s_range=(0, 1500))
    for ps in (big, small, small):
        t = _device_pairs(torch, ps)
        native.sw_batch_torch(t, mat, 12, 2)
        torch.cuda.synchronize()
        ref = np.stack([t[k].cpu().numpy() for k in _FIELDS])
        rc, got = _call_noalloc(torch, t, ps.n, mat, 12, 2)
        assert rc == 0
        assert (got == ref).all()


def test_noalloc_rejects_batches_above_its_limit(cuda):
    torch = cuda
    ps = synth.sw_pairs(MAX_PAIRS + 1, seed=8, q_range=(30, 60), s_range=(30, 60))
    t = _device_pairs(torch, ps)
    rc, got = _call_noalloc(torch, t, ps.n, synth.matrix("BLOSUM62"))
    assert rc == -4
    assert b"exceed" in native.lib().tpz_last_error()
    assert (got == -7).all()                          # nothing was written


def test_noalloc_matches_oracle_and_marks_long_queries_invalid(cuda):
    # checked against the CPU restatement of ssw_align directly, with queries
    # on both sides of the 1,024-residue limit of the fixed scratch
    import oracle
    torch = cuda
    mat = synth.matrix("BLOSUM62")
    ps = synth.sw_pairs(600, seed=91, q_median=900, q_range=(1, 1300), s_range=(0, 1200))
    t = _device_pairs(torch, ps)
    rc, got = _call_noalloc(torch, t, ps.n, mat)
    assert rc == 0, native.lib().tpz_last_error()
    long_q = ps.qlen > 1024
    assert long_q.sum() > 50 and (~long_q).sum() > 300
    assert (got[3][long_q] == native.TPZ_SW_INVALID).all()
    ok = np.flatnonzero(~long_q)
    ref = np.stack(oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, 11, 1))
    assert (got[:, ok] == ref[:, ok]).all()


def test_noalloc_rejects_matrices_beyond_16_bit_range(cuda):
    # largest entry 32: a 1,024-residue query could score past what the
    # 16-bit lanes hold exactly; 31 is still accepted and equals the
    # allocating call (which would re-run such scores in 32 bits)
    torch = cuda
    ps = synth.sw_pairs(300, seed=12, q_range=(900, 1024), s_range=(900, 1100))
    t = _device_pairs(torch, ps)
    for diag, want in ((32, -1), (31, 0)):
        mat = np.full((25, 25), -3, np.int8)
        np.fill_diagonal(mat, diag)
        rc, got = _call_noalloc(torch, t, ps.n, mat)
        assert rc == want, native.lib().tpz_last_error()
        if rc:
            assert b"largest matrix entry" in native.lib().tpz_last_error()
            assert (got == -7).all()
            continue
        native.sw_batch_torch(t, mat, 11, 1)
        torch.cuda.synchronize()
        ref = np.stack([t[k].cpu().numpy() for k in _FIELDS])
        assert (got == ref).all()
