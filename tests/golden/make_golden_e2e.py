"""End-to-end golden outputs of the UNMODIFIED reference `topaz` binary
(oracle/_ref/topaz): a seeded synthetic DB and query set, `topaz index`, then
`topaz search` in several modes.  python tests/golden/make_golden_e2e.py"""
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402
from topaz_b200 import synth  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "e2e")
MODES = {
    "default": [],
    "fast": ["--fast"],
    "blasttab": ["--blasttab"],
    "noseg": ["-M"],
    "b45": ["-m", "BLOSUM45", "-o", "14", "-e", "2", "-H", "20", "-E", "10"],
    "tight": ["-A", "60", "-S", "800", "-l", "6"],
}


def make_inputs():
    prot = synth.protein_db(600, seed=301)
    qs = synth.search_queries(prot, 30, 8, seed=302)
    rng = np.random.default_rng(303)
    ids, seqs = list(qs.ids), list(qs.seqs)
    for k, unit in enumerate((b"Q", b"PEST", b"GGS")):       # SEG targets
        core = np.frombuffer(unit * 30, np.uint8)
        src = prot.seqs[k * 7]
        ids.append("lc%d" % k)
        seqs.append(np.concatenate([src[:80], core, src[80:200]]))
    ids.append("short")
    seqs.append(np.frombuffer(b"MKV", np.uint8))
    synth.write_fasta(os.path.join(OUT, "db.fa"), prot)
    synth.write_fasta(os.path.join(OUT, "queries.fa"), synth.Proteins(ids, seqs))


if __name__ == "__main__":
    if oracle.libref() is None and not oracle.build_ref():
        sys.exit("the reference sources are needed to regenerate the fixtures")
    os.makedirs(OUT, exist_ok=True)
    make_inputs()
    work = "/tmp/tpz_e2e_ref"
    os.makedirs(work, exist_ok=True)
    pre = os.path.join(work, "db")
    subprocess.run([oracle.REF_BIN, "index", "-f", os.path.join(OUT, "db.fa"), "-p", pre],
                   check=True, capture_output=True)
    for name, extra in MODES.items():
        r = subprocess.run([oracle.REF_BIN, "search", "-f", os.path.join(OUT, "queries.fa"), "-p", pre,
                            "-T", "1", *extra], check=True, capture_output=True, cwd=work)
        with open(os.path.join(OUT, name + ".out"), "wb") as f:
            f.write(r.stdout)
        print(name, r.stdout.count(b"\n"))
