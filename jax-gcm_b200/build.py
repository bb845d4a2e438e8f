"""Builds ``libspeedy_b200.so`` in-tree with nvcc for sm_100a (no JIT cache, no torch ABI).

Each translation unit is compiled to an object in parallel, then linked into one shared
library; objects go to ``jax-gcm_b200/_build/`` (not committed).
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SOURCES = ["csrc/speedy_api.cu", "csrc/speedy_noalloc.cu", "csrc/speedy_ensemble.cu",
           "csrc/speedy_adjoint.cu"]
HEADERS = ["csrc/speedy_column.cuh", "csrc/speedy_column_smem.cuh", "csrc/speedy_derived.h",
           "csrc/speedy_kernels.cuh", "csrc/speedy_ad.h", "csrc/speedy_generic.h",
           "csrc/speedy_vjp.h",
           "../include/speedy_b200.h"]
OUT = os.path.join(HERE, "libspeedy_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def _nvcc():
    return os.environ.get("NVCC", "nvcc")


def compile_command(src, verbose=False):
    obj = os.path.join(OBJ_DIR, os.path.basename(src).replace(".cu", ".o"))
    cmd = [_nvcc(), *ARCH, *FLAGS, "-I" + os.path.join(ROOT, "include"), "-c",
           os.path.join(HERE, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    return cmd, obj


def nvcc_command(verbose=False):
    """The single-step equivalent of the build (documentation / reproduction)."""
    return [_nvcc(), *ARCH, *FLAGS, "-shared", "-I" + os.path.join(ROOT, "include"), "-o", OUT,
            *[os.path.join(HERE, s) for s in SOURCES]] + (["-Xptxas", "-v"] if verbose else [])


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in SOURCES + HEADERS)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    os.makedirs(OBJ_DIR, exist_ok=True)
    jobs = [compile_command(s, verbose) for s in SOURCES]

    def run(job):
        cmd, _ = job
        return cmd, subprocess.run(cmd, capture_output=True, text=True)

    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        results = list(ex.map(run, jobs))
    for cmd, res in results:
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
        if verbose:
            sys.stderr.write(res.stderr)
    link = [_nvcc(), *ARCH, "-shared", "-o", OUT, *[obj for _, obj in jobs]]
    res = subprocess.run(link, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc link failed: " + " ".join(link))
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
