"""TOPAZ database files: .pin / .psq / .phr / .ind / .SA / .ISA.

Layouts (written by ``demultiplex_fasta`` src/demux.c:15-50 and
``serif_index``/``create_index`` src/index.c:24-172):

* ``.psq``  internal-alphabet residues, each protein followed by '\\n';
* ``.phr``  one ID per line (header up to the first space or tab);
* ``.pin``  text lines ``psq_offset length phr_offset idlen``;
* ``.ind``  packed records {u64 header_start, u64 protein_start,
  i32 header_len, i32 protein_len} (24 bytes, src/db.h:10-17);
* ``.SA``   little-endian int64 suffix array over the bytes of ``.psq``;
* ``.ISA``  zero-filled file of the same size (only filled under USE_LCP).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

from . import alphabet as ab

IND_DTYPE = np.dtype([("header_start", "<u8"), ("protein_start", "<u8"),
                      ("header_len", "<i4"), ("protein_len", "<i4")])


@dataclass
class Database:
    T: np.ndarray          # uint8, internal alphabet + '\n'
    SA: np.ndarray | None  # int64
    ind: np.ndarray        # IND_DTYPE records
    headers: bytes

    @property
    def Tsize(self):
        return len(self.T)

    @property
    def Psize(self):
        return len(self.ind)

    @property
    def pstart(self):
        return self.ind["protein_start"].astype(np.int64)

    def protein_id(self, i):
        r = self.ind[i]
        return self.headers[int(r["header_start"]):int(r["header_start"]) + int(r["header_len"])]


def parse_fasta(data: bytes):
    """fasta_next/_create_seq (src/fasta.c:80-120, :62-78) record splitting.

    A record runs from a '>' that starts the file or follows '\\n' up to the
    next such '>'.  The ID is the header up to the first space/tab
    (src/seq.c:55-78); the residues are every non-'\\n' byte after the
    header line, upper-cased by upper_aa (src/seq.c:80-104)."""
    out = []
    n = len(data)
    if n == 0:
        return out
    starts = [0] + [i + 1 for i in range(n - 1) if data[i] == 10 and data[i + 1] == 62]
    bounds = starts[1:] + [n + 1]
    for st, nx in zip(starts, bounds):
        rec = data[st:nx - 1]
        nl = rec.find(b"\n")
        if nl < 0:
            raise ValueError("FASTA record without a newline")
        hdr = rec[:nl]
        h0 = 1 if hdr[:1] == b">" else 0
        idend = h0
        while idend < len(hdr) and hdr[idend] not in (32, 9):
            idend += 1
        seq = np.frombuffer(rec[nl + 1:], dtype=np.uint8)
        seq = seq[seq != 10]
        out.append((hdr[h0:idend], ab.upper_aa(seq)))
    return out


def build_from_records(records) -> Database:
    """T, .ind and .phr for (id, upper-case residues) records (demux.c:29-34)."""
    tparts, hparts, rows = [], [], []
    toff = hoff = 0
    for pid, seq in records:
        internal = ab.aa_to_internal(seq)
        rows.append((hoff, toff, len(pid), len(internal)))
        tparts.append(internal.tobytes() + b"\n")
        hparts.append(pid + b"\n")
        toff += len(internal) + 1
        hoff += len(pid) + 1
    T = np.frombuffer(b"".join(tparts), dtype=np.uint8).copy()
    ind = np.array(rows, dtype=IND_DTYPE)
    return Database(T, None, ind, b"".join(hparts))


def write_files(prefix: str, db: Database):
    with open(prefix + ".psq", "wb") as f:
        f.write(db.T.tobytes())
    with open(prefix + ".phr", "wb") as f:
        f.write(db.headers)
    with open(prefix + ".pin", "w") as f:
        for r in db.ind:
            f.write("%d %d %d %d\n" % (r["protein_start"], r["protein_len"],
                                       r["header_start"], r["header_len"]))
    with open(prefix + ".ind", "wb") as f:
        f.write(db.ind.tobytes())
    with open(prefix + ".SA", "wb") as f:
        f.write(np.ascontiguousarray(db.SA, dtype="<i8").tobytes())
    with open(prefix + ".ISA", "wb") as f:
        f.truncate(8 * db.Tsize)


def read_files(prefix: str) -> Database:
    T = np.fromfile(prefix + ".psq", dtype=np.uint8)
    SA = np.fromfile(prefix + ".SA", dtype="<i8")
    if len(SA) != len(T):
        raise ValueError("%s.SA holds %d entries, %s.psq %d bytes" % (prefix, len(SA), prefix, len(T)))
    headers = open(prefix + ".phr", "rb").read()
    nprot = headers.count(b"\n")
    ind = np.fromfile(prefix + ".ind", dtype=IND_DTYPE)
    if len(ind) != nprot:
        raise ValueError("%s.ind holds %d records, expected %d" % (prefix, len(ind), nprot))
    return Database(T, SA, ind, headers)


def exists(prefix: str) -> bool:
    return all(os.path.exists(prefix + e) for e in (".psq", ".SA", ".phr", ".ind"))


def build_from_arrays(residues: np.ndarray, lens: np.ndarray, id_prefix: str = "db") -> Database:
    """T, .ind and .phr for proteins given as concatenated upper-case residues
    and lengths (ids id_prefix0, id_prefix1, ...), without per-protein loops."""
    lens = np.asarray(lens, dtype=np.int64)
    n = len(lens)
    internal = ab.aa_to_internal(residues)
    pstart = np.cumsum(lens + 1) - (lens + 1)
    T = np.full(int(lens.sum()) + n, ord("\n"), dtype=np.uint8)
    pos = np.repeat(pstart - (np.cumsum(lens) - lens), lens) + np.arange(int(lens.sum()))
    T[pos] = internal
    ids = [("%s%d" % (id_prefix, i)).encode() for i in range(n)]
    hl = np.array([len(x) for x in ids], dtype=np.int64)
    hs = np.cumsum(hl + 1) - (hl + 1)
    ind = np.zeros(n, dtype=IND_DTYPE)
    ind["header_start"] = hs
    ind["protein_start"] = pstart
    ind["header_len"] = hl
    ind["protein_len"] = lens
    return Database(T, None, ind, b"\n".join(ids) + b"\n")
