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
           "csrc/speedy_adjoint.cu", "csrc/held_suarez.cu", "csrc/speedy_selftest.cu"]
HEADERS = ["csrc/speedy_column.cuh", "csrc/speedy_column_smem.cuh", "csrc/speedy_derived.h",
           "csrc/speedy_kernels.cuh", "csrc/speedy_ensemble.cuh", "csrc/speedy_ad.h",
           "csrc/speedy_generic.h", "csrc/speedy_vjp.h", "csrc/speedy_pk.cuh",
           "../include/speedy_b200.h"]
OUT = os.path.join(HERE, "libspeedy_b200.so")
OBJ_DIR = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]
# The forward kernels (speedy_ensemble.cu) are compiled without multiply-add contraction
# (-fmad=false): the reference's float32 arithmetic (XLA without fast-math, like NumPy) rounds
# every product and every sum, and contraction was the main source of the forward's elementwise
# distance to it (measured at T425: humidity tendency 7.2e-6 -> 2.8e-6 and convective
# precipitation 6.7e-6 -> 2.4e-6 of their maxima, wind tendencies 1e-6 -> 1.5e-8, downward
# shortwave 2.1e-4 -> 4.5e-5; it costs about 5 % of the forward's time).  They divide with the
# hardware's approximate division and flush subnormal results to zero: the forward is bound by
# instruction issue, IEEE division and subnormal handling cost several instructions each, and
# measured against the oracles they change nothing (tendencies, precipitation and diagnostics
# keep their distances at the printed digits; the only values flushed are transmissivities below
# 1e-38).  The adjoint keeps IEEE division and subnormals and is compiled without contraction
# too: its kernel exists in two register budgets (four or two blocks per SM, chosen by the
# batch's tile count), and only separately rounded arithmetic makes the two give the same bits,
# so that a member's gradients do not depend on the batch it is served in (with contraction
# ptxas fused different products in the two; without it the T170 VJP takes 0.566 against
# 0.529 ms, and the reference's float32 arithmetic rounds every operation as well).
FORWARD_FLAGS = ["-fmad=false", "-prec-div=false", "-ftz=true"]
SOURCE_FLAGS = {"csrc/speedy_ensemble.cu": FORWARD_FLAGS,
                "csrc/speedy_selftest.cu": FORWARD_FLAGS,  # checks the forward's arithmetic
                "csrc/speedy_adjoint.cu": ["-fmad=false"]}


def _nvcc():
    return os.environ.get("NVCC", "nvcc")


def compile_command(src, verbose=False):
    obj = os.path.join(OBJ_DIR, os.path.basename(src).replace(".cu", ".o"))
    cmd = [_nvcc(), *ARCH, *FLAGS, *SOURCE_FLAGS.get(src, []),
           "-I" + os.path.join(ROOT, "include"), "-c", os.path.join(HERE, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    return cmd, obj


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = SOURCES + HEADERS + [os.path.basename(__file__)]  # flags live in this file
    return any(os.path.getmtime(os.path.join(HERE, d)) > t for d in deps)


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
