"""Device query ingest (tpz_prepare_queries_device: SEG hard-masking + the
internal alphabet) equals the host's (tpz_prepare_queries, whose masks are
pinned to the reference's run_seg goldens) byte for byte: the reference's
golden inputs, low-complexity repeats of many kinds, mixtures with
non-standard residues, and the search-workload queries."""
import ctypes
import os

import numpy as np
import pytest

from topaz_b200 import alphabet as ab, native, synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _device_prepare(torch, queries, seg=True):
    L = native.lib()
    L.tpz_prepare_queries_device.argtypes = [ctypes.c_void_p] * 3 + [ctypes.c_int64] * 2 + \
        [ctypes.c_int, ctypes.c_void_p]
    lens = np.array([len(q) for q in queries], np.int32)
    off = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.int64)
    cat = np.frombuffer(b"".join(queries), np.uint8).copy()
    dev = torch.device("cuda:0")
    d_cat = torch.from_numpy(cat if len(cat) else np.zeros(1, np.uint8)).to(dev)
    d_off, d_len = torch.from_numpy(off).to(dev), torch.from_numpy(lens).to(dev)
    native.check(L.tpz_prepare_queries_device(d_cat.data_ptr(), d_off.data_ptr(), d_len.data_ptr(),
                                              len(queries), len(cat), 1 if seg else 0,
                                              torch.cuda.current_stream().cuda_stream))
    b = d_cat.cpu().numpy().tobytes()
    return [b[o:o + n] for o, n in zip(off.tolist(), lens.tolist())]


def _inputs():
    from test_host_parity import seg_inputs
    g = np.load(os.path.join(HERE, "golden", "seg_golden.npz"))
    offs = list(g["off"]) + [len(g["seqs"])]
    golden = [g["seqs"][a:b].tobytes() for a, b in zip(offs[:-1], offs[1:])]
    rng = np.random.default_rng(23)
    extra = []
    for k in range(300):        # short tandem repeats inside random sequence, both ends
        unit = synth.random_residues(rng, int(rng.integers(1, 6))).tobytes()
        core = unit * int(rng.integers(2, 80))
        extra.append(synth.random_residues(rng, int(rng.integers(0, 300))).tobytes() + core +
                     synth.random_residues(rng, int(rng.integers(0, 300))).tobytes())
    return golden + seg_inputs() + extra


@pytest.mark.parametrize("seg", [True, False])
def test_device_ingest_equals_host(cuda, seg):
    qs = _inputs()
    assert _device_prepare(cuda, qs, seg) == native.prepare_queries(qs, seg=seg)


def test_device_ingest_golden_masks(cuda):
    g = np.load(os.path.join(HERE, "golden", "seg_golden.npz"))
    offs = list(g["off"]) + [len(g["seqs"])]
    qs = [g["seqs"][a:b].tobytes() for a, b in zip(offs[:-1], offs[1:])]
    want = [ab.aa_to_internal(np.frombuffer(g["masked"][a:b].tobytes(), np.uint8)).tobytes()
            for a, b in zip(offs[:-1], offs[1:])]
    assert _device_prepare(cuda, qs) == want


def test_device_ingest_search_workload(cuda):
    res, lens = synth.protein_db_arrays(3000, seed=24)
    qres, qlens = synth.search_queries_arrays(res, lens, 1500, 1500, seed=25, lo=30, hi=3000)
    qoff = np.cumsum(qlens) - qlens
    qs = [qres[o:o + n].tobytes() for o, n in zip(qoff, qlens)]
    assert _device_prepare(cuda, qs) == native.prepare_queries(qs)


@pytest.mark.parametrize("ingest", [1, 2])
def test_search_batch_with_device_ingest(cuda, ingest):
    # raw residues into tpz_search_batch (SEG + alphabet on the device) give
    # the same hits as queries prepared on the host
    from sa_util import make_db
    prot = synth.protein_db(1500, seed=26)
    db = make_db(prot)
    raw = [bytes(s) for s in synth.search_queries(prot, 40, 20, seed=27, hi=3000).seqs]
    raw.append(b"QQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQQ" + raw[0])   # a masked run
    mat = synth.matrix("BLOSUM62")
    ix = native.Index(db)
    try:
        rep = {"max_evalue": 10.0, "stats": True}
        a = ix.search(native.prepare_queries(raw, seg=ingest == 1), mat, report=rep)
        b = ix.search(raw, mat, report=rep, ingest=ingest)
    finally:
        ix.close()
    for k in ("hit_off", "npops", "ncounted", "protein", "rawscore", "qend", "send", "evalue",
              "qstart", "sstart", "length", "gapopen", "mismatch"):
        assert np.array_equal(a[k], b[k]), k
    assert len(a["protein"]) > 40
