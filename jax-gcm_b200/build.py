"""Builds ``libspeedy_b200.so`` in-tree with nvcc for sm_100a (no JIT cache, no torch ABI)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["csrc/speedy_api.cu", "csrc/speedy_noalloc.cu", "csrc/speedy_ensemble.cu"]
HEADERS = ["csrc/speedy_column.cuh", "csrc/speedy_column_smem.cuh", "csrc/speedy_derived.h",
           "csrc/speedy_kernels.cuh",
           "../include/speedy_b200.h"]
OUT = os.path.join(HERE, "libspeedy_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_command(verbose=False):
    nvcc = os.environ.get("NVCC", "nvcc")
    cmd = [nvcc, *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-I" + os.path.join(ROOT, "include"), "-o", OUT]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    cmd += [os.path.join(HERE, s) for s in SOURCES]
    return cmd


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = SOURCES + HEADERS
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    cmd = nvcc_command(verbose)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if verbose:
        sys.stderr.write(res.stderr)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
