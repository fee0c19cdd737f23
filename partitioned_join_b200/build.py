"""Builds the native parts in-tree: partitioned_join_b200/libpj.so (the C ABI
of include/pj.h over the sm_100a kernels) and partitioned_join_b200/bin/
partitioned_join (the command-line drop-in for the reference binary).

    python -m partitioned_join_b200.build [--force]
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpj.so")
BIN_DIR = os.path.join(PKG, "bin")
CLI = os.path.join(BIN_DIR, "partitioned_join")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]

LIB_SOURCES = ["pj_api.cu", "pj_noalloc.cu", "pj_generate.cu", "pj_batch.cu", "pj_learn.cu"]


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cuh", ".h", ".cpp"))]
    cli_dir = os.path.join(CSRC, "cli")
    if os.path.isdir(cli_dir):
        files += [os.path.join(cli_dir, f) for f in os.listdir(cli_dir)]
    files.append(os.path.join(ROOT, "include", "pj.h"))
    return files


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> None:
    deps = _deps()
    if force or _stale(LIB, deps):
        cmd = [NVCC, *COMMON, "-shared", "-cudart", "static",
               *[os.path.join(CSRC, s) for s in LIB_SOURCES], "-o", LIB]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
    cli_src = os.path.join(CSRC, "cli", "partitioned_join_cli.cu")
    if os.path.exists(cli_src) and (force or _stale(CLI, deps + [cli_src, LIB])):
        os.makedirs(BIN_DIR, exist_ok=True)
        cmd = [NVCC, *COMMON, cli_src, "-o", CLI, "-L", PKG, "-lpj", "-Xlinker", "-rpath,$ORIGIN/..",
               "-cudart", "static"]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
