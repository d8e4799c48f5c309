"""`topaz search` on damaged database files, on the host: a .SA whose size is
not 8 x the .psq size and a .ind whose size is not 24 x the number of
proteins end the process with the reference's messages and exit status
(db_load/_load_index, src/db.c:61-64, :117-120) before any device work, so
these run without a GPU.  When the reference binary is built (oracle/_ref),
its stderr and status are compared line for line."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from topaz_b200 import build as B, dbformat, synth

from sa_util import make_db


@pytest.fixture(scope="module")
def dbfiles(tmp_path_factory):
    B.build()
    d = tmp_path_factory.mktemp("cli_host")
    prot = synth.protein_db(60, seed=7)
    db = make_db(prot)
    pre = str(d / "db")
    dbformat.write_files(pre, db)
    qs = synth.search_queries(prot, 3, 1, seed=8)
    qfa = str(d / "q.fa")
    synth.write_fasta(qfa, qs)
    return pre, qfa


def _damaged(pre, tmp_path, ext, keep):
    out = str(tmp_path / "bad")
    for e in (".psq", ".SA", ".phr", ".ind", ".pin"):
        data = open(pre + e, "rb").read()
        if e == ext:
            data = data[:keep(len(data))]
        open(out + e, "wb").write(data)
    return out


def _run(exe, qfa, pre):
    return subprocess.run([exe, "search", "-f", qfa, "-p", pre], capture_output=True,
                          cwd=os.path.dirname(pre), timeout=120)


@pytest.mark.parametrize("ext,keep,msg", [
    (".SA", lambda n: n - 8, b"should be 8 x T"),
    (".SA", lambda n: 0, b"could not load database, Invalid argument"),
    (".ind", lambda n: n - 24, b"index is the wrong size"),
    (".ind", lambda n: n - 1, b"index is the wrong size"),
])
def test_search_rejects_truncated_index_files(dbfiles, tmp_path, ext, keep, msg):
    pre, qfa = dbfiles
    bad = _damaged(pre, tmp_path, ext, keep)
    r = _run(B.CLI, qfa, bad)
    assert r.returncode == 1, r.stderr.decode()[-500:]
    assert msg in r.stderr
    assert r.stdout == b""
    if os.path.exists(oracle.REF_BIN):
        rr = _run(oracle.REF_BIN, qfa, bad)
        assert rr.returncode == r.returncode
        assert rr.stderr == r.stderr


def test_search_reports_missing_index_file(dbfiles, tmp_path):
    pre, qfa = dbfiles
    bad = _damaged(pre, tmp_path, ".SA", lambda n: n)
    os.remove(bad + ".ind")
    r = _run(B.CLI, qfa, bad)
    assert r.returncode == 1
    assert b"could not open" in r.stderr and b".ind" in r.stderr
    assert r.stderr.endswith(b"Error: could not load database, No such file or directory\n")
    if os.path.exists(oracle.REF_BIN):
        rr = _run(oracle.REF_BIN, qfa, bad)
        assert (rr.returncode, rr.stderr) == (r.returncode, r.stderr)
