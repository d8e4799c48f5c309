"""SEG golden vectors: run_seg of the unmodified reference (oracle/_ref) on
seeded sequences (random, tandem repeats, low-entropy mixtures with
non-standard residues).  python tests/golden/make_golden_seg.py"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
import oracle  # noqa: E402
from test_host_parity import seg_inputs  # noqa: E402

if __name__ == "__main__":
    R = oracle.libref()
    if R is None and not oracle.build_ref():
        sys.exit("the reference sources are needed to regenerate the fixtures")
    R = oracle.libref()
    R.ref_seg.argtypes = [ctypes.c_char_p, ctypes.c_int]
    seqs = seg_inputs()
    masked = []
    for s in seqs:
        b = ctypes.create_string_buffer(s, len(s))
        R.ref_seg(b, len(s))
        masked.append(b.raw[:len(s)])
    off = np.concatenate([[0], np.cumsum([len(s) for s in seqs])]).astype(np.int64)
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "seg_golden.npz"),
                        seqs=np.frombuffer(b"".join(seqs), np.uint8),
                        masked=np.frombuffer(b"".join(masked), np.uint8), off=off)
    print("masked residues:", sum(m.count(b"X") - s.count(b"X") for s, m in zip(seqs, masked)))
