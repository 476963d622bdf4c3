"""Builds the in-tree shared library libissl_b200.so (CUDA for sm_100a + host C++).

    python -m cracklingplusplus_gpu_b200.build        (or __graft_entry__.build())

nvcc compiles every source directly for sm_100a; the .so lands next to this file so it
travels with the source tree. The host compiler runs with -ffp-contract=off so the MIT table
is computed with the same operation order as the reference's formula.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libissl_b200.so")
CLI = os.path.join(HERE, "issl_score_offtargets")
EXTRACT_CLI = os.path.join(HERE, "issl_extract_offtargets")
SOURCES = ["index.cu", "score.cu", "radix_sort.cu", "synth.cu", "tables.cpp", "module.cpp", "tune.cpp", "serve.cpp", "extract.cu"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I" + os.path.join(REPO, "include"), "-I" + CSRC,
]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(REPO, "include", f) for f in os.listdir(os.path.join(REPO, "include"))]
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(objdir, src + ".o")
        cmd = [NVCC, *FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out))
        elif out and (verbose or ptxas_info):
            print(out)
    if failed:
        msg = "\n".join(f"--- {s}\n{o}" for s, o in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    tmp = LIB + ".tmp"
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp, *objs,
           "-Xcompiler", "-fPIC", "-lcudart"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    # the command-line mirror of ISSLScoreOfftargets, linked against the library
    cmd = [NVCC, *FLAGS, os.path.join(CSRC, "cli.cpp"), "-o", CLI + ".tmp", "-L" + HERE, "-lissl_b200",
           "-Xlinker", "-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    os.replace(CLI + ".tmp", CLI)
    # the command-line mirror of ExtractOfftargets
    cmd = [NVCC, *FLAGS, os.path.join(CSRC, "extract_cli.cpp"), "-o", EXTRACT_CLI + ".tmp", "-L" + HERE,
           "-lissl_b200", "-Xlinker", "-rpath,$ORIGIN"]
    subprocess.run(cmd, check=True)
    os.replace(EXTRACT_CLI + ".tmp", EXTRACT_CLI)
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
