"""Device --blasttab statistics (tpz_sw_stats_device) against the host
restatement (tpzh_align_stats, pinned to the reference) and the reference's
own ssw_align_stats (oracle/_ref): start coordinates, length, gap opens,
mismatches and identity of every aligned pair, bit for bit, over several
matrices and gap settings, homologous and random pairs, short and long."""
import ctypes

import numpy as np
import pytest

import oracle
from topaz_b200 import native, synth

pytestmark = pytest.mark.gpu
FIELDS = ("qstart", "sstart", "length", "gapopen", "mismatch")


class St(ctypes.Structure):
    _fields_ = [("qstart", ctypes.c_int32), ("sstart", ctypes.c_int32), ("length", ctypes.c_int32),
                ("mismatch", ctypes.c_int32), ("gapopen", ctypes.c_int32),
                ("identity", ctypes.c_double)]


def _device_stats(torch, ps, mat, go, ge, fwd):
    L = native.lib()
    vp = ctypes.c_void_p
    L.tpz_sw_stats_device.argtypes = [ctypes.c_int64] + [vp] * 7 + [ctypes.c_int, ctypes.c_int] + \
        [vp] * 10
    dev = torch.device("cuda:0")
    t = {k: torch.from_numpy(np.ascontiguousarray(getattr(ps, k))).to(dev)
         for k in ("q", "qoff", "qlen", "s", "soff", "slen")}
    sc, re_, rd = (torch.from_numpy(np.ascontiguousarray(x, np.int32)).to(dev) for x in fwd)
    out = {k: torch.full((ps.n,), -9, dtype=torch.int32, device=dev) for k in FIELDS}
    ident = torch.full((ps.n,), -9.0, dtype=torch.float64, device=dev)
    native.check(L.tpz_sw_stats_device(
        ps.n, *[t[k].data_ptr() for k in ("q", "qoff", "qlen", "s", "soff", "slen")],
        np.ascontiguousarray(mat, np.int8).ctypes.data, go, ge, rd.data_ptr(), re_.data_ptr(),
        sc.data_ptr(), *[out[k].data_ptr() for k in FIELDS], ident.data_ptr(),
        torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    res = {k: out[k].cpu().numpy() for k in FIELDS}
    res["identity"] = ident.cpu().numpy()
    return res


def _same_double(a, b):
    return (a == b) or (np.isnan(a) and np.isnan(b))


@pytest.mark.parametrize("name,go,ge,seed", [("BLOSUM62", 11, 1, 1), ("BLOSUM45", 14, 2, 2),
                                              ("PAM30", 9, 1, 3), ("BLOSUM62", 3, 1, 4)])
def test_device_stats_match_host_and_reference(cuda, name, go, ge, seed):
    torch = cuda
    mat = synth.matrix(name)
    ps = synth.sw_pairs(1500, seed=700 + seed, homolog_frac=0.7, q_range=(1, 1500),
                        s_range=(1, 2500))
    sc, re_, rd, st = native.sw_batch_host(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, go, ge)
    ok = st == native.TPZ_SW_OK
    got = _device_stats(torch, ps, mat, go, ge, (sc, re_, rd))
    L = native.lib()
    L.tpzh_align_stats.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(St)]
    R = oracle.libref()
    matc = np.ascontiguousarray(mat, np.int8)
    nref = 0
    for i in np.flatnonzero(ok):
        q = np.ascontiguousarray(ps.q[ps.qoff[i]:ps.qoff[i] + ps.qlen[i]], np.int8)
        s = np.ascontiguousarray(ps.s[ps.soff[i]:ps.soff[i] + ps.slen[i]], np.int8)
        h = St()
        L.tpzh_align_stats(q.ctypes.data, len(q), s.ctypes.data, len(s), matc.ctypes.data, go, ge,
                           int(rd[i]), int(re_[i]), int(sc[i]), ctypes.byref(h))
        mine = tuple(int(got[k][i]) for k in FIELDS)
        assert mine == tuple(getattr(h, k) for k in FIELDS), (i, mine)
        assert _same_double(got["identity"][i], h.identity), i
        if R is not None and i % 5 == 0:
            ref = [ctypes.c_int32() for _ in range(5)] + [ctypes.c_double()]
            R.ref_ssw_stats(oracle._p(q), ctypes.c_int32(len(q)), oracle._p(s), ctypes.c_int32(len(s)),
                            oracle._p(matc), go, ge, ctypes.c_int32(int(rd[i])),
                            ctypes.c_int32(int(re_[i])), ctypes.c_int32(int(sc[i])),
                            *[ctypes.byref(x) for x in ref])
            qs_, ss_, ln, gop, mm = (x.value for x in ref[:5])
            assert (int(got["qstart"][i]), int(got["sstart"][i]), int(got["length"][i]),
                    int(got["gapopen"][i]), int(got["mismatch"][i])) == (qs_, ss_, ln, gop, mm), i
            assert _same_double(got["identity"][i], ref[5].value), i
            nref += 1
    assert ok.sum() > 1000
    assert R is None or nref > 200


def test_device_stats_edge_pairs(cuda):
    # zero-score pairs (no end cell), one-residue queries, all-X pairs
    torch = cuda
    mat = synth.matrix("BLOSUM62")
    q = [np.array([0], np.int8), np.full(30, 23, np.int8), np.array([4, 4, 4], np.int8),
         np.arange(25, dtype=np.int8)]
    s = [np.array([0, 1, 0], np.int8), np.full(40, 23, np.int8), np.array([4], np.int8),
         np.arange(25, dtype=np.int8)[::-1].copy()]
    ps = synth.PairSet(np.concatenate(q), np.cumsum([0] + [len(x) for x in q[:-1]]).astype(np.int64),
                       np.array([len(x) for x in q], np.int32), np.concatenate(s),
                       np.cumsum([0] + [len(x) for x in s[:-1]]).astype(np.int64),
                       np.array([len(x) for x in s], np.int32), 0)
    sc, re_, rd, st = native.sw_batch_host(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, 11, 1)
    got = _device_stats(torch, ps, mat, 11, 1, (sc, re_, rd))
    L = native.lib()
    for i in range(ps.n):
        h = St()
        L.tpzh_align_stats(ps.q[ps.qoff[i]:].ctypes.data, int(ps.qlen[i]), ps.s[ps.soff[i]:].ctypes.data,
                           int(ps.slen[i]), np.ascontiguousarray(mat, np.int8).ctypes.data, 11, 1,
                           int(rd[i]), int(re_[i]), int(sc[i]), ctypes.byref(h))
        assert tuple(int(got[k][i]) for k in FIELDS) == tuple(getattr(h, k) for k in FIELDS), i
        assert _same_double(got["identity"][i], h.identity), i
