"""INTEGRATION.md's engine-side snippet is the code of
oracle/integration_example.c (compiled against the TOPAZ headers by
`make -C oracle relink`), so the documented code is code that compiles."""
import os
import re
import subprocess

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _snippet():
    src = open(os.path.join(ROOT, "oracle", "integration_example.c")).read()
    a = src.index("/* BEGIN INTEGRATION SNIPPET */\n") + len("/* BEGIN INTEGRATION SNIPPET */\n")
    return src[a:src.index("/* END INTEGRATION SNIPPET */")]


def test_integration_doc_holds_the_compiled_snippet():
    doc = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    blocks = re.findall(r"```c\n(.*?)```", doc, re.S)
    assert _snippet() in blocks


@pytest.mark.skipif(not oracle.REF_SRC or not os.path.isdir(oracle.REF_SRC),
                    reason="TOPAZ sources not present (TOPAZ_REF_SRC)")
def test_integration_snippet_compiles_against_reference_headers(tmp_path):
    out = str(tmp_path / "snippet.o")
    subprocess.run(["gcc", "-O2", "-Wall", "-Werror", "-Wno-unused-function", "-I",
                    os.path.join(ROOT, "include"), "-I", oracle.REF_SRC, "-I",
                    os.path.join(oracle.REF_SRC, "seg"), "-c",
                    os.path.join(ROOT, "oracle", "integration_example.c"), "-o", out], check=True)
