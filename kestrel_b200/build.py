"""Builds libkestrel_gpu.so (sm_100a) and the `kestrel` CLI in-tree with nvcc.

The library lands next to this file so that it travels with the repository;
nothing is installed into site-packages.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libkestrel_gpu.so")
CLI = os.path.join(HERE, "bin", "kestrel")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CUDA_SOURCES = ["kg_engine.cu", "kg_wave.cu", "kg_api.cu", "kg_noalloc.cu", "kg_soft.cu", "kg_multi.cu"]
HOST_SOURCES = ["kg_cli.cpp", "kg_vcf.cpp"]
HEADERS = ["kg_engine.h", "kg_pair.cuh", "kg_solver.cuh", "kg_rowsolve.cuh", "kg_wave.cuh", "kg_bulk.cuh",
           "kg_vcf.h", "kg_threads.h", "kg_allele.cuh", "kg_alleleN.cuh", "kg_qp1.cuh"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    nv = nvcc()
    common = ["-O3", "-std=c++17", "-lineinfo", "-I", INCLUDE, "-I", CSRC, "-Xcompiler", "-fPIC"]
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "kestrel_gpu.h")]
    objs = []
    for src in CUDA_SOURCES + HOST_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            flags = common + (ARCH + ["-Xptxas", "-v"] if src.endswith(".cu") else ["-x", "cu"] + ARCH)
            r = _run([nv] + flags + ["-c", s, "-o", o])
            if verbose:
                sys.stderr.write(r.stderr)
    if force or _newer(LIB, objs):
        _run([nv] + ARCH + ["-shared", "-o", LIB] + objs + ["-lz"])
    main = os.path.join(CSRC, "kg_main.cpp")
    if force or _newer(CLI, [main, LIB]):
        _run([nv] + ["-O2", "-std=c++17", "-I", INCLUDE, main, "-o", CLI, "-L", HERE, "-lkestrel_gpu",
                     "-Xlinker", "-rpath=$ORIGIN/.."])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
