"""Suffix array construction on the device (tpz_sa_build, used by
`topaz index`): equal to a CPU suffix array on random, repetitive and tiny
texts, and `topaz index` writes the reference's .SA bytes."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import oracle
from sa_util import suffix_array
from topaz_b200 import alphabet as ab, build as B, dbformat, native, synth

pytestmark = pytest.mark.gpu


def _sa(T):
    L = native.lib()
    L.tpz_sa_build.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p]
    T = np.ascontiguousarray(T, dtype=np.uint8)
    SA = np.empty(max(len(T), 1), np.int64)
    rounds = ctypes.c_int32()
    native.check(L.tpz_sa_build(T.ctypes.data, len(T), SA.ctypes.data, ctypes.byref(rounds)))
    return SA[:len(T)], rounds.value


def _text(prot):
    recs = [(pid.encode(), ab.upper_aa(s)) for pid, s in zip(prot.ids, prot.seqs)]
    return dbformat.build_from_records(recs).T


def test_sa_build_random_and_repetitive_texts(cuda):
    prot = synth.protein_db(2000, seed=71)
    T = _text(prot)
    SA, r = _sa(T)
    assert np.array_equal(SA, suffix_array(T))
    # the same proteins three times over: long common prefixes, more rounds
    T3 = np.concatenate([T, T, T])
    SA3, r3 = _sa(T3)
    assert np.array_equal(SA3, suffix_array(T3))
    assert r3 > r
    # one letter repeated: every suffix a prefix of the next longer one
    Ta = np.frombuffer(b"A" * 5000 + b"\n", np.uint8)
    SAa, _ = _sa(Ta)
    assert np.array_equal(SAa, suffix_array(Ta))


SINK = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                        ctypes.POINTER(ctypes.c_int64), ctypes.c_int64)


def _sa_sink(T, max_partition):
    """tpz_sa_build_sink with a sink that records every piece it is given."""
    L = native.lib()
    L.tpz_sa_build_sink.argtypes = [ctypes.c_void_p, ctypes.c_int64, SINK, ctypes.c_void_p,
                                    ctypes.c_int64, ctypes.c_void_p]
    T = np.ascontiguousarray(T, dtype=np.uint8)
    SA = np.full(len(T), -1, np.int64)
    pieces = []

    def sink(user, first, rows, count):
        SA[first:first + count] = np.ctypeslib.as_array(rows, shape=(count,))
        pieces.append((first, count))
        return 0

    cb = SINK(sink)
    rounds = ctypes.c_int32()
    native.check(L.tpz_sa_build_sink(T.ctypes.data, len(T), cb, None, max_partition,
                                     ctypes.byref(rounds)))
    return SA, pieces, rounds.value


@pytest.mark.parametrize("max_partition", [0, 50_000, 3_000])
def test_sa_build_partitions_and_doubling(cuda, max_partition):
    # many partitions (a cap on the suffixes sorted at once), repeats long
    # enough for the doubling phase, and rows delivered piece by piece
    prot = synth.protein_db(1500, seed=73)
    T = _text(prot)
    Tr = np.concatenate([T, T[:20000], T, np.frombuffer(b"M" * 2080 + b"\n", np.uint8)])
    SA, pieces, r = _sa_sink(Tr, max_partition)
    assert np.array_equal(SA, suffix_array(Tr))
    covered = np.zeros(len(Tr), bool)
    for a, c in pieces:
        covered[a:a + c] = True
    assert covered.all()
    if max_partition:
        assert len(pieces) > len(Tr) // max_partition


def test_sa_build_wide_alphabet(cuda):
    # arbitrary bytes (more than 32 distinct values: 6 bits per symbol)
    rng = np.random.default_rng(74)
    T = rng.integers(0, 200, 30000).astype(np.uint8)
    T[5000:9000] = T[1000:5000]
    SA, _ = _sa(T)
    assert np.array_equal(SA, suffix_array(T))


@pytest.mark.parametrize("text", [b"\n", b"A\n", b"AA", b"BA\nAB\n", b"YYYYYYYYYY\nYYYYYYYYY\n"])
def test_sa_build_tiny_texts(cuda, text):
    T = np.frombuffer(text, np.uint8)
    SA, _ = _sa(T)
    assert np.array_equal(SA, suffix_array(T))


def test_sa_build_empty(cuda):
    SA, r = _sa(np.zeros(0, np.uint8))
    assert len(SA) == 0 and r == 0


@pytest.mark.skipif(not os.path.exists(oracle.REF_BIN), reason="reference binary not built")
def test_topaz_index_writes_the_reference_sa(cuda, tmp_path):
    prot = synth.protein_db(3000, seed=72)
    fa = os.path.join(str(tmp_path), "db.fa")
    synth.write_fasta(fa, prot)
    outs = {}
    for who, exe in (("ref", oracle.REF_BIN), ("mine", B.CLI)):
        pre = os.path.join(str(tmp_path), who)
        r = subprocess.run([exe, "index", "-f", fa, "-p", pre], check=True, capture_output=True)
        if who == "mine":
            assert b"suffix array construction failed" not in r.stderr
        outs[who] = {e: open(pre + e, "rb").read() for e in (".psq", ".SA", ".ind", ".pin", ".phr")}
    for e in outs["ref"]:
        assert outs["ref"][e] == outs["mine"][e], e
