import ctypes

import numpy as np
import pytest

import oracle
from sa_util import suffix_array
from topaz_b200 import synth, dbformat


def test_suffix_array_sorted_small():
    T = np.frombuffer(b"BANANA\nBAN\nANA\n", dtype=np.uint8)
    sa = suffix_array(T)
    sufs = [T[i:].tobytes() for i in sa]
    assert sufs == sorted(sufs)
    assert sorted(sa.tolist()) == list(range(len(T)))


@pytest.mark.skipif(oracle.libref() is None, reason="oracle/_ref not built")
def test_suffix_array_equals_divsufsort():
    prot = synth.protein_db(300, seed=9)
    db = dbformat.build_from_records([(p.encode(), s) for p, s in zip(prot.ids, prot.seqs)])
    ref = np.zeros(db.Tsize, np.int64)
    assert oracle.libref().divsufsort64(oracle._p(db.T), oracle._p(ref), ctypes.c_int64(db.Tsize)) == 0
    assert (suffix_array(db.T) == ref).all()
