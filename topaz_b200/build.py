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
SOURCES = ["tpz_common.cu", "sw_kernel.cu", "search_kernels.cu", "search_host.cu", "sa_build.cu", "ssw_shim.cu",
           "stats_kernel.cu", "seg_kernel.cu"]
# per-file nvcc flags: the device SEG must round every double operation
# separately (no fused multiply-adds), as the host code does
EXTRA_FLAGS = {"seg_kernel.cu": ["-fmad=false"]}
HOSTDIR = os.path.join(HERE, "host")
HOST_SOURCES = ["tpzh_fasta.c", "tpzh_seg.c", "tpzh_index.c", "tpzh_stats.c",
                "tpzh_search.c", "tpzh_main.c", "tpzh_prepare.c"]
CLI = os.path.join(LIBDIR, "topaz")
CC = os.environ.get("CC", "gcc")
# plain IEEE double arithmetic in the host code (no fast-math, no FMA
# contraction) so that SEG and E-values round exactly as the reference does
HOST_CFLAGS = ["-O2", "-g", "-fPIC", "-std=gnu11", "-Wall", "-Wno-unused-result",
               "-fvisibility=hidden", "-ffp-contract=off"]


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
    deps += [os.path.join(HOSTDIR, f) for f in os.listdir(HOSTDIR) if f.endswith((".c", ".h"))]
    deps.append(os.path.join(ROOT, "include", "topaz_b200.h"))
    if not force and not _stale(LIB, deps) and not _stale(CLI, deps):
        return LIB
    objs = []
    procs = []
    for src in sources():
        obj = os.path.join(LIBDIR, os.path.basename(src) + ".o")
        cmd = [NVCC, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
               "--default-stream", "per-thread",
               "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj,
               *EXTRA_FLAGS.get(os.path.basename(src), [])]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT), src))
        objs.append(obj)
    for src in HOST_SOURCES:
        obj = os.path.join(LIBDIR, src + ".o")
        cmd = [CC, *HOST_CFLAGS, "-I", os.path.join(ROOT, "include"), "-c",
               os.path.join(HOSTDIR, src), "-o", obj]
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
    link = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xlinker", "-Bsymbolic", "-lm", "-lpthread"]
    subprocess.check_call(link)
    cli = [CC, "-O2", "-o", CLI, os.path.join(HOSTDIR, "tpzh_cli.c"), "-I", HOSTDIR, "-L", LIBDIR,
           "-ltopaz_b200", "-Wl,-rpath,$ORIGIN", "-lm"]
    subprocess.check_call(cli)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
