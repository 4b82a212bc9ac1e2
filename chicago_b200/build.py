"""Build the in-tree CUDA library chicago_b200/libevxg.so for sm_100a.

Usage: python -m chicago_b200.build [--verbose]

The library is compiled by nvcc directly (no torch extension, no JIT cache):
every kernel is sm_100a-only (-gencode arch=compute_100a,code=sm_100a), with
-fmad=false so no floating-point contraction can change an RD cost.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libevxg.so")
SOURCES = ["evxg_mb.cu", "evxg_filters.cu", "evxg_api.cu", "evxg_batch.cu", "evxg_serve.cu", "evxg_noalloc.cu", "evxg_decode.cu",
           "evxg_serialize.cpp", "evxg_mux.cpp"]
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")


def nvcc_cmd(verbose: bool = False):
    cmd = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
           "-fmad=false", "-Xcompiler", "-fPIC,-O2", "-shared", "-I", os.path.join(ROOT, "include"),
           "-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES] + ["-lcudart"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    return cmd


def up_to_date() -> bool:
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "evxg.h")]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    if force or not up_to_date():
        r = subprocess.run(nvcc_cmd(verbose), capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError("nvcc failed building libevxg.so")
    return LIB


if __name__ == "__main__":
    build(force=True, verbose="--verbose" in sys.argv)
    print(LIB)
