"""Host-side pieces of the CLI against the reference (CPU only):
SEG masking, the suffix array, `topaz index` files, blasttab statistics,
bitscores and E-values."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from topaz_b200 import build as B, native, synth

HERE = os.path.dirname(os.path.abspath(__file__))
needs_ref = pytest.mark.skipif(oracle.libref() is None, reason="oracle/_ref not built")


def host():
    L = native.lib()
    L.tpzh_seg_mask.argtypes = [ctypes.c_char_p, ctypes.c_int]
    return L


def seg_inputs():
    rng = np.random.default_rng(17)
    out = []
    aa = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWY", np.uint8)
    for n in (5, 11, 12, 13, 30, 100, 400, 1500):
        out.append(synth.random_residues(rng, n).tobytes())
    for unit in (b"Q", b"QQN", b"AP", b"SGS", b"PEST", b"KKE", b"GGGGS"):
        for reps in (3, 8, 40, 200):
            core = unit * reps
            left = synth.random_residues(rng, int(rng.integers(0, 60))).tobytes()
            right = synth.random_residues(rng, int(rng.integers(0, 60))).tobytes()
            out.append(left + core + right)
    for k in range(60):        # low-entropy mixtures incl. non-standard residues
        n = int(rng.integers(12, 600))
        alph = aa[rng.choice(20, size=int(rng.integers(1, 5)), replace=False)]
        seq = alph[rng.integers(0, len(alph), n)]
        seq[rng.random(n) < 0.05] = ord("X")
        if k % 3 == 0:
            seq[rng.random(n) < 0.03] = int(rng.choice(list(b"BZUO*")))
        pre = synth.random_residues(rng, int(rng.integers(0, 100)))
        out.append(np.concatenate([pre, seq, synth.random_residues(rng, 20)]).tobytes())
    return out


def test_seg_matches_golden():
    g = np.load(os.path.join(HERE, "golden", "seg_golden.npz"))
    L = host()
    seqs, masked = g["seqs"].tobytes(), g["masked"].tobytes()
    off = g["off"]
    for i in range(len(off) - 1):
        s = bytearray(seqs[off[i]:off[i + 1]])
        buf = ctypes.create_string_buffer(bytes(s), len(s))
        L.tpzh_seg_mask(buf, len(s))
        assert buf.raw[:len(s)] == masked[off[i]:off[i + 1]], i


def test_prepare_queries_batch_matches_golden_seg():
    """tpz_prepare_queries (SEG + internal alphabet over host threads) on the
    golden SEG inputs equals SEG then the alphabet query by query."""
    from topaz_b200 import alphabet as ab, native
    g = np.load(os.path.join(HERE, "golden", "seg_golden.npz"))
    seqs, masked = g["seqs"].tobytes(), g["masked"].tobytes()
    off = g["off"]
    qs = [seqs[off[i]:off[i + 1]] for i in range(len(off) - 1)]
    want = [ab.aa_to_internal(np.frombuffer(masked[off[i]:off[i + 1]], np.uint8)).tobytes()
            for i in range(len(off) - 1)]
    for threads in (1, 3, 16):
        assert native.prepare_queries(qs, threads=threads) == want
    nos = native.prepare_queries(qs, seg=False, threads=2)
    assert nos == [ab.aa_to_internal(np.frombuffer(q, np.uint8)).tobytes() for q in qs]
    assert native.prepare_queries([]) == []


@needs_ref
def test_seg_matches_live_reference():
    L, R = host(), oracle.libref()
    R.ref_seg.argtypes = [ctypes.c_char_p, ctypes.c_int]
    rng = np.random.default_rng(99)
    for s in seg_inputs() + [synth.random_residues(rng, 3000).tobytes()]:
        a = ctypes.create_string_buffer(s, len(s))
        b = ctypes.create_string_buffer(s, len(s))
        R.ref_seg(a, len(s))
        L.tpzh_seg_mask(b, len(s))
        assert a.raw[:len(s)] == b.raw[:len(s)]


def _fasta_cases(tmp):
    prot = synth.protein_db(120, seed=4)
    path = os.path.join(tmp, "db.fa")
    synth.write_fasta(path, prot)
    quirky = os.path.join(tmp, "quirky.fa")
    with open(quirky, "wb") as f:
        f.write(b">p1 desc\tmore\nacdefGHIKL\nMNPQ\r\n>p2\n\n>>p3 x\nBZUOJ*x-\n>p4\tt\nWWW\n>p5\nAC")
    return [path, quirky]


@needs_ref
@pytest.mark.gpu
def test_index_files_match_reference(cuda, tmp_path):
    # `topaz index` builds the suffix array on the device
    B.build()
    for fa in _fasta_cases(str(tmp_path)):
        outs = {}
        for who, exe in (("ref", oracle.REF_BIN), ("mine", B.CLI)):
            pre = os.path.join(str(tmp_path), who + os.path.basename(fa))
            subprocess.run([exe, "index", "-f", fa, "-p", pre], check=True, capture_output=True)
            outs[who] = {e: open(pre + e, "rb").read() for e in (".pin", ".psq", ".phr", ".ind", ".SA", ".ISA")}
        for e in outs["ref"]:
            assert outs["ref"][e] == outs["mine"][e], (fa, e)


@needs_ref
def test_blasttab_stats_match_reference():
    L, R = host(), oracle.libref()

    class St(ctypes.Structure):
        _fields_ = [("qstart", ctypes.c_int32), ("sstart", ctypes.c_int32), ("length", ctypes.c_int32),
                    ("mismatch", ctypes.c_int32), ("gapopen", ctypes.c_int32), ("identity", ctypes.c_double)]
    L.tpzh_align_stats.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int32,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int32,
                                   ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(St)]
    ps = synth.sw_pairs(400, seed=12, homolog_frac=0.7, q_range=(20, 900), s_range=(20, 1500))
    for name, go, ge in (("BLOSUM62", 11, 1), ("BLOSUM45", 14, 2), ("PAM30", 9, 1)):
        mat = synth.matrix(name)
        sc, re_, rd, stt = oracle.reference_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, go, ge)
        n = 0
        for i in range(ps.n):
            if stt[i] != 0 or sc[i] < 30:
                continue
            q = np.ascontiguousarray(ps.q[ps.qoff[i]:ps.qoff[i] + ps.qlen[i]])
            s = np.ascontiguousarray(ps.s[ps.soff[i]:ps.soff[i] + ps.slen[i]])
            o = [ctypes.c_int32() for _ in range(5)] + [ctypes.c_double()]
            R.ref_ssw_stats(oracle._p(q), ctypes.c_int32(len(q)), oracle._p(s), ctypes.c_int32(len(s)),
                            oracle._p(mat), go, ge, ctypes.c_int32(rd[i]), ctypes.c_int32(re_[i]),
                            ctypes.c_int32(sc[i]), *[ctypes.byref(x) for x in o])
            m = St()
            L.tpzh_align_stats(q.ctypes.data, len(q), s.ctypes.data, len(s), mat.ctypes.data, go, ge,
                               int(rd[i]), int(re_[i]), int(sc[i]), ctypes.byref(m))
            ref = (o[0].value, o[1].value, o[2].value, o[4].value, o[3].value)
            mine = (m.qstart, m.sstart, m.length, m.mismatch, m.gapopen)
            assert ref == mine, (name, i, ref, mine)
            assert np.float64(o[5].value).tobytes() == np.float64(m.identity).tobytes()
            n += 1
        assert n > 100


@pytest.mark.parametrize("variant", ["default", "tight"])
def test_karlin_matches_reference_golden(golden_search, variant):
    # bitscore and E-value of every aligned hit (gapless >= 40 goes through
    # ssw_align; no golden hit reaches the 16-bit drop) as exact doubles
    g = golden_search
    hi, hf, meta = g["hitsi_" + variant], g["hitsf_" + variant], g["meta_" + variant]
    ind = g["ind"].view(np.uint8)
    nprot = len(ind) // 24
    db_size = len(g["T"]) - nprot
    h0, checked = 0, 0
    for q in range(len(g["qlen"])):
        nh = int(meta[q][2])
        for j in range(h0, h0 + nh):
            if hi[j, 2] == 1 and hi[j, 1] >= 40:
                bits, ev = native.karlin(int(g["qlen"][q]), db_size, nprot, int(hi[j, 3]))
                assert (ev, bits) == (hf[j, 0], hf[j, 1]), (q, j, hi[j], hf[j])
                checked += 1
        h0 += nh
    assert checked > 20
