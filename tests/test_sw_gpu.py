"""GPU parity of the batched Smith-Waterman kernel (through the C ABI).

Bit-exact against: the reference's golden vectors (ssw_init + ssw_align
outputs on seeded pairs, tests/golden/sw_golden.npz) and the oracle on fresh
seeded pairs; at the full microbench size (10^6 pairs) through a random
oracle-checked sample plus batch-order independence."""
import numpy as np
import pytest

import oracle
from topaz_b200 import native, synth

pytestmark = pytest.mark.gpu


def _settings(g):
    for k in g:
        if k.count("_") == 2 and not k.startswith("mat_"):
            name, go, ge = k.split("_")
            yield k, g["mat_" + name], int(go), int(ge)


def _to_dev(torch, ps):
    d = torch.device("cuda:0")
    t = {"q": torch.from_numpy(np.ascontiguousarray(ps.q)).to(d),
         "qoff": torch.from_numpy(ps.qoff).to(d), "qlen": torch.from_numpy(ps.qlen).to(d),
         "s": torch.from_numpy(np.ascontiguousarray(ps.s)).to(d),
         "soff": torch.from_numpy(ps.soff).to(d), "slen": torch.from_numpy(ps.slen).to(d)}
    n = len(ps.qlen)
    for k in ("score", "ref_end", "read_end", "status"):
        t[k] = torch.full((n,), -7, dtype=torch.int32, device=d)
    return t


def _run_dev(torch, ps, mat, go=11, ge=1):
    t = _to_dev(torch, ps)
    native.sw_batch_torch(t, mat, go, ge)
    torch.cuda.synchronize()
    return np.stack([t[k].cpu().numpy() for k in ("score", "ref_end", "read_end", "status")])


def test_sw_host_api_matches_reference_golden(cuda, golden_sw):
    g = golden_sw
    for key, mat, go, ge in _settings(g):
        got = np.stack(native.sw_batch_host(g["q"], g["qoff"], g["qlen"], g["s"], g["soff"],
                                            g["slen"], mat, go, ge))
        bad = np.flatnonzero((got != g[key]).any(axis=0))
        assert bad.size == 0, (key, bad[:5], got[:, bad[:5]], g[key][:, bad[:5]])


def test_sw_device_api_matches_reference_golden(cuda, golden_sw):
    g = golden_sw
    ps = synth.PairSet(g["q"], g["qoff"], g["qlen"], g["s"], g["soff"], g["slen"], 0)
    for key, mat, go, ge in _settings(g):
        got = _run_dev(cuda, ps, mat, go, ge)
        assert (got == g[key]).all(), key


@pytest.mark.parametrize("seed,go,ge,name", [(1, 11, 1, "BLOSUM62"), (2, 12, 2, "BLOSUM50"),
                                             (3, 9, 1, "PAM30"), (4, 10, 1, "BLOSUM90"),
                                             (5, 14, 2, "PAM250")])
def test_sw_matches_oracle_fresh_pairs(cuda, seed, go, ge, name):
    ps = synth.sw_pairs(6000, seed=seed, q_range=(1, 1024), s_range=(0, 4000))
    mat = synth.matrix(name)
    got = _run_dev(cuda, ps, mat, go, ge)
    ref = np.stack(oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat, go, ge))
    bad = np.flatnonzero((got != ref).any(axis=0))
    assert bad.size == 0, (bad[:5], got[:, bad[:5]], ref[:, bad[:5]], ps.qlen[bad[:5]], ps.slen[bad[:5]])


def test_sw_every_row_bin_and_odd_batch(cuda):
    # one pair per query length 1..1024 (all 32 row bins, ragged tails, an odd
    # pair count so one task carries a single pair)
    rng = np.random.default_rng(9)
    qs = [rng.integers(0, 20, L).astype(np.int8) for L in range(1, 1025)]
    ss = [np.concatenate([q[::-1][: rng.integers(1, len(q) + 1)], rng.integers(0, 20, 50).astype(np.int8)])
          for q in qs]
    qs.append(rng.integers(0, 20, 333).astype(np.int8)); ss.append(np.zeros(0, np.int8))
    ql = np.array([len(x) for x in qs], np.int32); sl = np.array([len(x) for x in ss], np.int32)
    qo = np.concatenate([[0], np.cumsum(ql)[:-1]]).astype(np.int64)
    so = np.concatenate([[0], np.cumsum(sl)[:-1]]).astype(np.int64)
    ps = synth.PairSet(np.concatenate(qs), qo, ql, np.concatenate(ss), so, sl, 0)
    mat = synth.matrix("BLOSUM62")
    got = _run_dev(cuda, ps, mat)
    ref = np.stack(oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat))
    assert (got == ref).all()



def test_sw_short_subjects_and_wavefront_edges(cuda):
    # every lane computes every step, before its first column and past the
    # subject's end: subjects of 0-2 columns, around the 32-column wavefront
    # fill and the 32-step refresh, next to queries on and around the
    # stripe and lane-segment boundaries; random, self and strongly
    # homologous content (the latter saturates the u8 pass), in one batch so
    # short and long subjects share bins and tasks
    rng = np.random.default_rng(31)
    qs, ss = [], []
    for ql in (1, 2, 31, 32, 33, 96, 352, 1000, 1024, 1025):
        q = rng.integers(0, 20, ql).astype(np.int8)
        for sl in (0, 1, 2, 31, 32, 33, 63, 64, 65, 97, 500):
            qs.append(q); ss.append(rng.integers(0, 20, sl).astype(np.int8))
            qs.append(q); ss.append(np.resize(q, sl).astype(np.int8))
    ql = np.array([len(x) for x in qs], np.int32); sl = np.array([len(x) for x in ss], np.int32)
    qo = np.concatenate([[0], np.cumsum(ql)[:-1]]).astype(np.int64)
    so = np.concatenate([[0], np.cumsum(sl)[:-1]]).astype(np.int64)
    s_all = np.concatenate(ss) if sl.sum() else np.zeros(0, np.int8)
    ps = synth.PairSet(np.concatenate(qs), qo, ql, s_all, so, sl, 0)
    mat = synth.matrix("BLOSUM62")
    got = _run_dev(cuda, ps, mat)
    ref = np.stack(oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat))
    bad = np.flatnonzero((got != ref).any(axis=0))
    assert bad.size == 0, (bad[:5], got[:, bad[:5]], ref[:, bad[:5]], ps.qlen[bad[:5]], ps.slen[bad[:5]])
    assert (ref[0] + 4 >= 255).any()                 # some pairs took the i16 pass
    host = np.stack(native.sw_batch_host(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat))
    assert (host == ref).all()

def test_sw_full_size_sample_and_order_independence(cuda):
    ps = synth.sw_pairs(1_000_000, seed=1)
    mat = synth.matrix("BLOSUM62")
    got = _run_dev(cuda, ps, mat)
    assert (got[3] == native.TPZ_SW_OK).all()
    rng = np.random.default_rng(0)
    idx = rng.choice(ps.n, 4000, replace=False)
    sub = synth.PairSet(ps.q, ps.qoff[idx], ps.qlen[idx], ps.s, ps.soff[idx], ps.slen[idx], 0)
    ref = np.stack(oracle.oracle_sw(sub.q, sub.qoff, sub.qlen, sub.s, sub.soff, sub.slen, mat))
    assert (got[:, idx] == ref).all()
    # the same pairs in reverse order give the same per-pair results
    rev = np.arange(ps.n)[::-1].copy()
    psr = synth.PairSet(ps.q, ps.qoff[rev], ps.qlen[rev], ps.s, ps.soff[rev], ps.slen[rev], 0)
    got_r = _run_dev(cuda, psr, mat)
    assert (got_r[:, ::-1] == got).all()


def test_sw_host_large_batch_matches_device(cuda):
    # the host entry point on 160 MB of residues equals the device call on
    # the same pairs, in any pair order, and on pairs that share a subject
    ps = synth.sw_pairs(200_000, seed=8)
    assert len(ps.q) + len(ps.s) > 64 << 20
    mat = synth.matrix("BLOSUM62")
    dev = _run_dev(cuda, ps, mat)
    host = np.stack(native.sw_batch_host(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat))
    assert (host == dev).all()
    perm = np.random.default_rng(2).permutation(ps.n)
    hp = np.stack(native.sw_batch_host(ps.q, ps.qoff[perm], ps.qlen[perm], ps.s, ps.soff[perm],
                                       ps.slen[perm], mat))
    assert (hp == dev[:, perm]).all()
    # every pair aligned against the last subject
    last = np.full(1000, ps.n - 1)
    hl = np.stack(native.sw_batch_host(ps.q, ps.qoff[:1000], ps.qlen[:1000], ps.s,
                                       ps.soff[last], ps.slen[last], mat))
    idx = np.arange(1000)
    sub = synth.PairSet(ps.q, ps.qoff[idx], ps.qlen[idx], ps.s, ps.soff[last], ps.slen[last], 0)
    ref = np.stack(oracle.oracle_sw(sub.q, sub.qoff, sub.qlen, sub.s, sub.soff, sub.slen, mat))
    assert (hl == ref).all()


def test_sw_long_queries_multi_stripe(cuda):
    # queries longer than one 1024-row stripe: random, homologous (u8
    # saturation -> i16 pass) and W-runs near / past the 16-bit limit (the
    # 32-bit rerun): 2977 W = 32747 (kept), 3000 W = 33000 (dropped)
    rng = np.random.default_rng(21)
    W = 17  # W in ARNDCQEGHILKMFPSTWYVBJZX*
    qs, ss = [], []
    for L in (1025, 1500, 2048, 2049, 3000, 4100):
        q = rng.integers(0, 20, L).astype(np.int8)
        qs.append(q); ss.append(rng.integers(0, 20, int(rng.integers(1, 1500))).astype(np.int8))
        qs.append(q); ss.append(np.concatenate([rng.integers(0, 20, 30).astype(np.int8), q[100:900]]))
    for L in (2900, 2977, 3000):
        q = np.full(L, W, np.int8)
        qs.append(q); ss.append(q.copy())
    ps = synth.sw_pairs(60, seed=3, q_range=(1025, 8192), q_median=2500, s_range=(0, 3000))
    qs += [ps.q[o:o + l] for o, l in zip(ps.qoff, ps.qlen)]
    ss += [ps.s[o:o + l] for o, l in zip(ps.soff, ps.slen)]
    # and short pairs in the same batch
    short = synth.sw_pairs(300, seed=4)
    qs += [short.q[o:o + l] for o, l in zip(short.qoff, short.qlen)]
    ss += [short.s[o:o + l] for o, l in zip(short.soff, short.slen)]
    ql = np.array([len(x) for x in qs], np.int32); sl = np.array([len(x) for x in ss], np.int32)
    qo = np.concatenate([[0], np.cumsum(ql)[:-1]]).astype(np.int64)
    so = np.concatenate([[0], np.cumsum(sl)[:-1]]).astype(np.int64)
    ps = synth.PairSet(np.concatenate(qs), qo, ql, np.concatenate(ss), so, sl, 0)
    mat = synth.matrix("BLOSUM62")
    got = _run_dev(cuda, ps, mat)
    ref = np.stack(oracle.oracle_sw(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat))
    bad = np.flatnonzero((got != ref).any(axis=0))
    assert bad.size == 0, (bad[:5], got[:, bad[:5]], ref[:, bad[:5]], ps.qlen[bad[:5]])
    assert (ref[0] == 32747).any() and (ref[3] == native.TPZ_SW_DROPPED).any()
    host = np.stack(native.sw_batch_host(ps.q, ps.qoff, ps.qlen, ps.s, ps.soff, ps.slen, mat))
    assert (host == ref).all()


def test_sw_align_one_matches_reference_golden(cuda, golden_sw):
    """The per-pair launch form (tpz_sw_align_one) gives the reference's
    ssw_align results pair by pair, saturating u8 passes included."""
    torch = cuda
    g = golden_sw
    d = torch.device("cuda:0")
    q = torch.from_numpy(np.ascontiguousarray(g["q"])).to(d)
    s = torch.from_numpy(np.ascontiguousarray(g["s"])).to(d)
    n = len(g["qlen"])
    for key, mat, go, ge in _settings(g):
        out = torch.full((n, 4), -7, dtype=torch.int32, device=d)
        st = torch.cuda.current_stream().cuda_stream
        for i in range(n):
            native.sw_align_one(q.data_ptr() + int(g["qoff"][i]), g["qlen"][i],
                                s.data_ptr() + int(g["soff"][i]), g["slen"][i], mat, go, ge,
                                out.data_ptr() + 16 * i, st)
        torch.cuda.synchronize()
        got = out.cpu().numpy().T
        bad = np.flatnonzero((got != g[key]).any(axis=0))
        assert bad.size == 0, (key, bad[:5], got[:, bad[:5]], g[key][:, bad[:5]])


def test_sw_align_one_rejects_out_of_range(cuda):
    torch = cuda
    out = torch.zeros(4, dtype=torch.int32, device="cuda:0")
    q = torch.zeros(2048, dtype=torch.int8, device="cuda:0")
    mat = synth.matrix("BLOSUM62")
    with pytest.raises(native.TopazError):
        native.sw_align_one(q.data_ptr(), 1025, q.data_ptr(), 10, mat, 11, 1, out.data_ptr())
    with pytest.raises(native.TopazError):
        native.sw_align_one(q.data_ptr(), 10, q.data_ptr(), 10, mat, 1, 1, out.data_ptr())
