"""The native library loads without a GPU and exports every symbol that
include/*.h declares; argument checks happen before any device work."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from topaz_b200 import native, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        for m in re.finditer(r"TPZ_API\s+[\w\s\*]+?\b(\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "tpz_sw_batch_device" in names and "tpz_sw_batch_host" in names
    assert len(names) >= 6


def test_library_exports_every_declared_symbol():
    L = native.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_matrices_match_reference_tables(golden_sw):
    for name in ("BLOSUM62", "BLOSUM45", "PAM30", "BLOSUM80"):
        assert (native.matrix(name).ravel() == golden_sw["mat_" + name]).all()
    for name in ("BLOSUM50", "BLOSUM90", "PAM70", "PAM250"):
        assert native.matrix(name).shape == (25, 25)
    assert (native.matrix("BLOSUM62") == synth.matrix("BLOSUM62")).all()


def test_unknown_matrix_is_an_error():
    with pytest.raises(native.TopazError) as e:
        native.matrix("BLOSUM99")
    assert e.value.code == -1


def test_sw_rejects_bad_gaps_and_sizes_before_device_work():
    q = np.zeros(4, np.int8)
    with pytest.raises(native.TopazError) as e:
        native.sw_batch_host(q, [0], [4], q, [0], [4], synth.matrix(), 1, 1)
    assert e.value.code in (-1,)                      # gap_open <= gap_extend
    with pytest.raises(native.TopazError) as e:
        native.sw_batch_host(np.zeros(9000, np.int8), [0], [9000], q, [0], [4], synth.matrix())
    assert e.value.code == -4                         # qlen above the limit


def test_sw_host_names_the_first_bad_pair_of_a_large_batch():
    # a batch the host entry point cuts into chunks and scans in pieces on
    # several threads: the error names the first invalid pair, whichever
    # piece finds it first
    n = 300_000
    q = np.zeros(64, np.int8)
    qlen = np.full(n, 8, np.int32)
    qlen[250_001] = 0
    qlen[70_123] = 9000
    qlen[140_000] = -1
    with pytest.raises(native.TopazError) as e:
        native.sw_batch_host(q, np.zeros(n, np.int64), qlen, q, np.zeros(n, np.int64),
                             np.full(n, 8, np.int32), synth.matrix())
    assert e.value.code == -4
    assert "pair 70123 " in str(e.value)
