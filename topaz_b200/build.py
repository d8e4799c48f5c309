"""Builds libtopaz_b200.so (all CUDA sources, sm_100a) in-tree.

    python -m topaz_b200.build [--verbose]

The library is plain CUDA runtime + C ABI (include/topaz_b200.h); it does not
link against torch.  Output: topaz_b200/lib/libtopaz_b200.so.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libtopaz_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = ["tpz_common.cu", "sw_kernel.cu", "search_kernels.cu", "search_host.cu"]


def sources():
    return [os.path.join(CSRC, s) for s in SOURCES]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    deps = sources() + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                        if f.endswith((".cuh", ".h", ".inc"))]
    deps.append(os.path.join(ROOT, "include", "topaz_b200.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(LIBDIR, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
               "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    failed = False
    for p, src in procs:
        out, _ = p.communicate()
        if out and (verbose or p.returncode):
            sys.stderr.write(out.decode())
        if p.returncode:
            failed = True
            sys.stderr.write("nvcc failed on %s\n" % src)
    if failed:
        raise RuntimeError("building libtopaz_b200.so failed")
    link = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "-Bsymbolic"]
    subprocess.check_call(link)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
