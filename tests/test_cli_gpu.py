"""End to end through the `topaz` command line on the GPU: our `topaz index`
files, then `topaz search` output compared per query block with the
reference binary's output (golden files; live when oracle/_ref is built).
The reference prints query blocks in thread completion order, so blocks are
compared as a mapping qseqid -> ordered lines, plus the header line."""
import os
import subprocess

import pytest

import oracle
from topaz_b200 import build as B, synth

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "e2e")
MODES = {
    "default": [],
    "fast": ["--fast"],
    "blasttab": ["--blasttab"],
    "noseg": ["-M"],
    "b45": ["-m", "BLOSUM45", "-o", "14", "-e", "2", "-H", "20", "-E", "10"],
    "tight": ["-A", "60", "-S", "800", "-l", "6"],
}


def blocks(text: bytes):
    lines = text.decode().splitlines()
    out = {}
    for ln in lines[1:]:
        out.setdefault(ln.split("\t", 1)[0], []).append(ln)
    return lines[0] if lines else "", out


@pytest.fixture(scope="module")
def indexed(tmp_path_factory):
    B.build()
    d = tmp_path_factory.mktemp("e2e")
    pre = str(d / "db")
    subprocess.run([B.CLI, "index", "-f", os.path.join(GOLD, "db.fa"), "-p", pre], check=True,
                   capture_output=True)
    return pre


@pytest.mark.parametrize("mode", list(MODES))
def test_cli_search_matches_reference_golden(cuda, indexed, mode):
    r = subprocess.run([B.CLI, "search", "-f", os.path.join(GOLD, "queries.fa"), "-p", indexed,
                        *MODES[mode]], capture_output=True)
    assert r.returncode == 0, r.stderr.decode()[-2000:]
    want = open(os.path.join(GOLD, mode + ".out"), "rb").read()
    assert blocks(r.stdout) == blocks(want)


@pytest.mark.skipif(not os.path.exists(oracle.REF_BIN), reason="reference binary not built")
@pytest.mark.parametrize("extra", [[], ["--blasttab"], ["--fast", "-H", "50", "-E", "1"]])
def test_cli_search_matches_live_reference(cuda, tmp_path, extra):
    B.build()
    prot = synth.protein_db(4000, seed=401)
    qs = synth.search_queries(prot, 60, 20, seed=402, hi=3000)
    db_fa, q_fa = str(tmp_path / "db.fa"), str(tmp_path / "q.fa")
    synth.write_fasta(db_fa, prot)
    synth.write_fasta(q_fa, qs)
    outs = []
    for exe in (oracle.REF_BIN, B.CLI):
        pre = str(tmp_path / ("db_" + os.path.basename(exe)))
        subprocess.run([exe, "index", "-f", db_fa, "-p", pre], check=True, capture_output=True)
        r = subprocess.run([exe, "search", "-f", q_fa, "-p", pre, "-T", "4", *extra],
                           capture_output=True, cwd=str(tmp_path))
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        outs.append(blocks(r.stdout))
    assert outs[0] == outs[1]
    assert sum(len(v) for v in outs[0][1].values()) > 50


@pytest.mark.parametrize("extra", [[], ["--blasttab"]])
def test_cli_concurrent_batches_print_the_single_thread_output(cuda, tmp_path, extra):
    # -T 3 with batches of 7 queries keeps three batches in flight on the
    # device; the lines come out byte for byte as with one thread
    B.build()
    prot = synth.protein_db(3000, seed=411)
    qs = synth.search_queries(prot, 50, 25, seed=412, hi=2000)
    db_fa, q_fa = str(tmp_path / "db.fa"), str(tmp_path / "q.fa")
    synth.write_fasta(db_fa, prot)
    synth.write_fasta(q_fa, qs)
    pre = str(tmp_path / "db")
    subprocess.run([B.CLI, "index", "-f", db_fa, "-p", pre], check=True, capture_output=True)
    outs = []
    for args in (["-T", "1"], ["-T", "3", "--batch", "7"], ["-T", "4", "--batch", "1"]):
        r = subprocess.run([B.CLI, "search", "-f", q_fa, "-p", pre, *args, *extra], capture_output=True)
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        outs.append(r.stdout)
    assert outs[0] == outs[1] == outs[2]
    assert outs[0].count(b"\n") > 50
