"""Seeded synthetic workloads with the shapes of the TOPAZ benchmark configs.

No public dataset is involved: every residue is drawn from a fixed
``numpy.random.Generator(PCG64(seed))``.

* Background residues are i.i.d. from the Robinson & Robinson (1991, PNAS
  88:8880) amino-acid frequencies (the table NCBI BLAST uses).
* Mutated homologues substitute residue a by b with the BLOSUM62-implied
  conditional P(b | a, b != a) proportional to q_ab = p_a p_b exp(lambda s_ab),
  lambda solving sum p_a p_b exp(lambda s_ab) = 1 under those frequencies,
  and add geometric-length insertions and deletions.
* Lengths are log-normal with the stated median (sigma 0.6) clipped to the
  stated range.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass

import numpy as np

from . import alphabet as ab

# Robinson & Robinson background frequencies (per mille), 20 amino acids
_RR = {
    "A": 78.05, "C": 19.25, "D": 53.64, "E": 62.95, "F": 38.56, "G": 73.77,
    "H": 21.99, "I": 51.42, "K": 57.44, "L": 90.19, "M": 22.43, "N": 44.87,
    "P": 52.03, "Q": 42.64, "R": 51.29, "S": 71.20, "T": 58.41, "V": 64.41,
    "W": 13.30, "Y": 32.16,
}
AA20 = np.frombuffer("".join(sorted(_RR)).encode(), dtype=np.uint8)
P20 = np.array([_RR[chr(c)] for c in AA20], dtype=np.float64)
P20 /= P20.sum()

_MATRIX_FILE = os.path.join(os.path.dirname(__file__), "csrc", "tpz_matrices.inc")
_MATRICES: dict[str, np.ndarray] = {}


def matrix(name: str = "BLOSUM62") -> np.ndarray:
    """25x25 int8 table (row = subject letter, column = query letter) in the
    order ARNDCQEGHILKMFPSTWYVBJZX*."""
    if not _MATRICES:
        text = open(_MATRIX_FILE).read()
        for blk in re.finditer(r"TPZ_MATRIX_TEXT_(\w+)\[\] =((?:\s*\"[^\"]*\")+);", text):
            lines = re.findall(r"\"([^\"]*)\"", blk.group(2))
            rows = [ln.replace("\\n", "").split()[1:] for ln in lines[1:]]
            _MATRICES[blk.group(1)] = np.array(rows, dtype=np.int8).reshape(25, 25)
    return _MATRICES[name]


def _lambda(m20: np.ndarray, p: np.ndarray) -> float:
    lo, hi = 1e-3, 2.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        v = (np.outer(p, p) * np.exp(mid * m20)).sum()
        if v > 1.0:
            hi = mid
        else:
            lo = mid
    return 0.5 * (lo + hi)


_SUB_CACHE = {}


def _substitution_table():
    """Per amino acid a (index into AA20): cumulative P(b | a, b != a)."""
    if "t" not in _SUB_CACHE:
        m = matrix("BLOSUM62")
        idx = ab.aa_to_index(AA20).astype(np.int64)
        m20 = m[np.ix_(idx, idx)].astype(np.float64)
        lam = _lambda(m20, P20)
        q = np.outer(P20, P20) * np.exp(lam * m20)
        np.fill_diagonal(q, 0.0)
        q /= q.sum(axis=1, keepdims=True)
        _SUB_CACHE["t"] = np.cumsum(q, axis=1)
    return _SUB_CACHE["t"]


def lognormal_lengths(rng, n, median, lo, hi, sigma=0.6):
    x = rng.lognormal(np.log(median), sigma, size=n)
    return np.clip(np.rint(x), lo, hi).astype(np.int64)


# background residues are drawn through a 65536-entry table holding each amino
# acid round(65536 * p) times (largest-remainder rounding; |error| < 2e-5)
def _draw_table():
    raw = P20 * 65536
    cnt = np.floor(raw).astype(np.int64)
    rem = raw - cnt
    cnt[np.argsort(-rem)[: 65536 - cnt.sum()]] += 1
    return np.repeat(AA20, cnt)


_DRAW = _draw_table()


def random_residues(rng, n) -> np.ndarray:
    """n background residues as upper-case amino-acid bytes."""
    return _DRAW[rng.integers(0, 65536, size=n, dtype=np.uint16)]


def mutate_batch(rng, seqs: np.ndarray, lens: np.ndarray, identity: np.ndarray,
                 indel_rate: float = 0.02, indel_p: float = 0.5):
    """Mutates the concatenated sequences `seqs` (segment lengths `lens`) in
    one vectorised pass.  Each residue of segment i is substituted with
    probability 1 - identity[i] (BLOSUM62 conditional); then at rate
    `indel_rate` per position an insertion (random residues placed before
    it) or a deletion (of it and the following residues of its segment) of
    geometric(indel_p) length.  Returns (residues, new segment lengths)."""
    lens = np.asarray(lens, dtype=np.int64)
    n = int(lens.sum())
    seg = np.repeat(np.arange(len(lens)), lens)
    seg_end = np.cumsum(lens)[seg]
    cum = _substitution_table()
    pos = np.searchsorted(AA20, seqs)
    out = seqs.copy()
    sub = rng.random(n) > np.asarray(identity, dtype=np.float64)[seg]
    if sub.any():
        u = rng.random(int(sub.sum()))
        rows = cum[pos[sub]]
        out[sub] = AA20[np.minimum((rows < u[:, None]).sum(axis=1), 19)]
    if indel_rate <= 0 or n == 0:
        return out, lens.copy()
    ev = np.flatnonzero(rng.random(n) < indel_rate)
    ln = rng.geometric(indel_p, size=len(ev)).astype(np.int64)
    ins = rng.random(len(ev)) < 0.5
    # deletions: positions [e, min(e + ln, segment end)) removed
    diff = np.zeros(n + 1, dtype=np.int64)
    de, dl = ev[~ins], ln[~ins]
    np.add.at(diff, de, 1)
    np.add.at(diff, np.minimum(de + dl, seg_end[de]), -1)
    keep = np.cumsum(diff[:n]) == 0
    # insertions: ln random residues before position e
    ins_len = np.zeros(n, dtype=np.int64)
    np.add.at(ins_len, ev[ins], ln[ins])
    counts = ins_len + keep
    total = int(counts.sum())
    start = np.cumsum(counts) - counts
    res = random_residues(rng, total)
    kp = np.flatnonzero(keep)
    res[start[kp] + ins_len[kp]] = out[kp]
    new_lens = np.bincount(seg, weights=counts, minlength=len(lens)).astype(np.int64)
    return res, new_lens


def mutate(rng, seq: np.ndarray, identity: float, indel_rate: float = 0.02,
           indel_p: float = 0.5) -> np.ndarray:
    """One sequence through mutate_batch."""
    out, _ = mutate_batch(rng, seq, np.array([len(seq)]), np.array([identity]), indel_rate,
                          indel_p)
    return out


# ---------------------------------------------------------------- SW pairs

@dataclass
class PairSet:
    """Concatenated query/subject residues (matrix indices) with offsets."""
    q: np.ndarray       # int8, all queries concatenated
    qoff: np.ndarray    # int64
    qlen: np.ndarray    # int32
    s: np.ndarray       # int8, all subjects concatenated
    soff: np.ndarray    # int64
    slen: np.ndarray    # int32
    seed: int

    @property
    def n(self):
        return len(self.qlen)

    @property
    def cells(self):
        return int((self.qlen.astype(np.int64) * self.slen.astype(np.int64)).sum())


def _segment_positions(starts: np.ndarray, lens: np.ndarray) -> np.ndarray:
    """Concatenation of arange(starts[i], starts[i] + lens[i])."""
    lens = np.asarray(lens, dtype=np.int64)
    total = int(lens.sum())
    first = np.cumsum(lens) - lens
    return np.repeat(np.asarray(starts, dtype=np.int64) - first, lens) + np.arange(total)


def sw_pairs(n: int, seed: int = 1, q_median=350, q_range=(30, 1000), s_median=350,
             s_range=(30, 5000), homolog_frac=0.2, identity=(0.25, 0.60)) -> PairSet:
    """The batched Smith-Waterman microbench workload: n independent pairs,
    log-normal query/subject lengths, `homolog_frac` of subjects mutated from
    their query (identity uniform in `identity`, centred in background
    residues up to the sampled subject length, cut to the subject range),
    the rest background."""
    rng = np.random.Generator(np.random.PCG64(seed))
    qlen = lognormal_lengths(rng, n, q_median, *q_range)
    slen = lognormal_lengths(rng, n, s_median, *s_range)
    hom = rng.random(n) < homolog_frac
    q_aa = random_residues(rng, int(qlen.sum()))
    qoff = np.cumsum(qlen) - qlen
    hid = np.flatnonzero(hom)
    final_len = slen.copy()
    if len(hid):
        core, raw_len = mutate_batch(rng, q_aa[_segment_positions(qoff[hid], qlen[hid])],
                                     qlen[hid], rng.uniform(*identity, size=len(hid)))
        raw_off = np.cumsum(raw_len) - raw_len
        core_len = np.minimum(raw_len, s_range[1])
        hl = np.maximum(slen[hid], np.maximum(core_len, s_range[0]))
        final_len[hid] = hl
    soff = np.cumsum(final_len) - final_len
    s_aa = random_residues(rng, int(final_len.sum()))
    if len(hid):
        left = (hl - core_len) // 2
        s_aa[_segment_positions(soff[hid] + left, core_len)] = \
            core[_segment_positions(raw_off, core_len)]
    return PairSet(ab.aa_to_index(q_aa), qoff.astype(np.int64), qlen.astype(np.int32),
                   ab.aa_to_index(s_aa), soff.astype(np.int64), final_len.astype(np.int32), seed)


# ---------------------------------------------------------- protein DBs

@dataclass
class Proteins:
    ids: list
    seqs: list          # upper-case amino-acid byte arrays


def protein_db(n: int, seed: int = 0, median=300, lo=50, hi=2000) -> Proteins:
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = lognormal_lengths(rng, n, median, lo, hi)
    allres = random_residues(rng, int(lens.sum()))
    seqs, off = [], 0
    for ln in lens:
        seqs.append(allres[off:off + ln])
        off += int(ln)
    return Proteins([f"db{i}" for i in range(n)], seqs)


def search_queries(db: Proteins, n_mut: int, n_rand: int, seed: int = 2,
                   identity=(0.30, 0.70), lo=None, hi=None) -> Proteins:
    """Queries mutated from randomly chosen DB entries plus random decoys."""
    rng = np.random.Generator(np.random.PCG64(seed))
    ids, seqs = [], []
    for i in range(n_mut):
        src = db.seqs[int(rng.integers(len(db.seqs)))]
        q = mutate(rng, src, rng.uniform(*identity))
        if lo is not None and len(q) < lo:
            q = np.concatenate([q, random_residues(rng, lo - len(q))])
        if hi is not None:
            q = q[:hi]
        ids.append(f"mut{i}")
        seqs.append(q)
    for i in range(n_rand):
        ln = int(lognormal_lengths(rng, 1, 300, lo or 50, hi or 2000)[0])
        ids.append(f"rand{i}")
        seqs.append(random_residues(rng, ln))
    return Proteins(ids, seqs)


def write_fasta(path: str, prot: Proteins, width: int = 60):
    with open(path, "wb") as f:
        for pid, s in zip(prot.ids, prot.seqs):
            f.write(b">" + pid.encode() + b" synthetic\n")
            b = s.tobytes()
            for i in range(0, len(b), width):
                f.write(b[i:i + width] + b"\n")


def protein_db_arrays(n: int, seed: int = 0, median=300, lo=50, hi=2000):
    """(residues uint8 AA letters concatenated, lengths int64) of an n-protein
    DB, drawn like protein_db but without per-protein arrays."""
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = lognormal_lengths(rng, n, median, lo, hi)
    return random_residues(rng, int(lens.sum())), lens


def search_queries_arrays(res, lens: np.ndarray, n_mut: int, n_rand: int,
                          seed: int = 2, identity=(0.30, 0.90), lo=50, hi=1500):
    """Queries for the full-search configs: n_mut mutated from random DB
    proteins (identity uniform in `identity`, indels at 0.02), n_rand random,
    lengths clipped to [lo, hi].  `res` is the DB's concatenated residues, or
    a function giving the concatenated residues of a list of protein
    numbers.  Returns (residues, lengths)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    off = np.cumsum(lens) - lens
    pick = rng.integers(0, len(lens), n_mut)
    src = res(pick) if callable(res) else res[_segment_positions(off[pick], lens[pick])]
    mres, mlen = mutate_batch(rng, src, lens[pick], rng.uniform(*identity, size=n_mut))
    rlen = lognormal_lengths(rng, n_rand, 300, lo, hi)
    rres = random_residues(rng, int(rlen.sum()))
    # clip / pad the mutated ones to [lo, hi]
    moff = np.cumsum(mlen) - mlen
    keep = np.minimum(mlen, hi)
    parts, plens = [], []
    for o, k in zip(moff, keep):
        s = mres[o:o + k]
        if len(s) < lo:
            s = np.concatenate([s, random_residues(rng, lo - len(s))])
        parts.append(s)
        plens.append(len(s))
    allres = np.concatenate(parts + [rres])
    return allres, np.concatenate([np.array(plens, np.int64), rlen])


FASTA_ID_DIGITS = 9


def _db_fasta_chunk(args):
    """Worker: one chunk of records of write_db_fasta, written at its offset."""
    path, seed, k, a, lens, rec_off, prefix = args
    lens = np.asarray(lens, dtype=np.int64)
    pre = (">" + prefix).encode()
    hw = len(pre) + FASTA_ID_DIGITS + 1
    rec = hw + lens + 1
    start = np.concatenate([[0], np.cumsum(rec)[:-1]])
    rng = np.random.Generator(np.random.PCG64([seed, k]))
    # residues drawn for every byte of the chunk; the header and newline
    # bytes are then written over them, so each sequence stays i.i.d.
    buf = random_residues(rng, int(rec.sum()))
    for j, c in enumerate(pre):
        buf[start + j] = c
    num = np.arange(a, a + len(lens), dtype=np.int64)
    for j in range(FASTA_ID_DIGITS):
        buf[start + len(pre) + FASTA_ID_DIGITS - 1 - j] = ord("0") + (num // 10 ** j) % 10
    buf[start + hw - 1] = ord("\n")
    buf[start + hw + lens] = ord("\n")
    fd = os.open(path, os.O_WRONLY)
    try:
        mv = memoryview(buf)
        done = 0
        while done < len(buf):
            done += os.pwrite(fd, mv[done:], rec_off + done)
    finally:
        os.close(fd)
    return len(buf)


def write_db_fasta(path: str, n: int, seed: int = 0, median=300, lo=50, hi=2000,
                   id_prefix: str = "db", chunk: int = 1_000_000, workers: int = 0):
    """An n-protein DB with the lengths and residue model of protein_db_arrays
    written straight to FASTA (IDs id_prefix + 9 digits, one sequence line
    per record), chunk by chunk in `workers` processes -- for DBs of 10^7 to
    10^8 proteins that should not sit in memory twice.  Returns (lens,
    seq_start): the sequence lengths and the file offset of each sequence,
    so that callers can read proteins back from the file."""
    import multiprocessing as mp
    rng = np.random.Generator(np.random.PCG64(seed))
    lens = lognormal_lengths(rng, n, median, lo, hi)
    hw = len(id_prefix) + 2 + FASTA_ID_DIGITS
    rec = hw + lens + 1
    rec_start = np.concatenate([[0], np.cumsum(rec)[:-1]])
    total = int(rec.sum())
    with open(path, "wb") as f:
        f.truncate(total)
    jobs = [(path, seed, k, a, lens[a:a + chunk], int(rec_start[a]), id_prefix)
            for k, a in enumerate(range(0, n, chunk))]
    workers = workers or min(len(jobs), os.cpu_count() or 1)
    if workers <= 1:
        for j in jobs:
            _db_fasta_chunk(j)
    else:
        with mp.get_context("spawn").Pool(workers) as pool:
            pool.map(_db_fasta_chunk, jobs)
    return lens, rec_start + hw


def fasta_residues(mm, seq_start: np.ndarray, lens: np.ndarray, pick) -> np.ndarray:
    """Residues of records `pick` of a FASTA written by write_db_fasta
    (mm: its bytes, e.g. an np.memmap), concatenated."""
    if len(pick) == 0:
        return np.zeros(0, np.uint8)
    return np.concatenate([np.asarray(mm[seq_start[i]:seq_start[i] + lens[i]]) for i in pick])

