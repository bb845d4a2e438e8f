"""The compiled CPU restatement of the reference physics (oracle/cpu_port.cpp): the benchmark's
timed CPU baseline and reference arm.

BENCHMARK AND TEST INFRASTRUCTURE ONLY: ``bench.py`` (its cpu_baseline and ``--impl reference``
legs) and ``tests/`` load it; the CUDA product path never does.  ``build()`` compiles it with
g++ (-O3, OpenMP, no fast-math) into ``oracle/_build/``.
"""
from __future__ import annotations

import ctypes as C
import importlib
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "cpu_port.cpp")
HEADERS = [os.path.join(ROOT, "jax-gcm_b200", "csrc", h)
           for h in ("speedy_generic.h", "speedy_ad.h")] + [
    os.path.join(ROOT, "include", "speedy_b200.h")]
OUT = os.path.join(HERE, "_build", "libcpu_port.so")
FLAGS = ["-O3", "-fopenmp", "-std=c++17", "-shared", "-fPIC"]

_F = ("u", "v", "t", "q", "phi", "psa", "sst", "stl", "soilw", "snowc", "sice", "alb0",
      "fmask", "orog", "phis0", "sia", "coa")
_O = ("du", "dv", "dt", "dq", "precnv", "precls", "cloudc", "rsds", "rlds")


class Instance_t(C.Structure):
    _fields_ = ([("kx", C.c_int), ("ix", C.c_int), ("il", C.c_int), ("flags", C.c_uint32),
                 ("model_step", C.c_int), ("tyear", C.c_float), ("ablco2", C.c_float)] +
                [(n, C.c_void_p) for n in _F] + [(n, C.c_void_p) for n in _O] +
                [("iptop", C.c_void_p), ("icltop", C.c_void_p)])


def command():
    return ["g++", *FLAGS, "-I" + os.path.join(ROOT, "include"),
            "-I" + os.path.join(ROOT, "jax-gcm_b200", "csrc"), "-o", OUT, SRC]


def build(force=False):
    """Compiles the CPU port if it is missing or older than its sources."""
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(p) <= t for p in [SRC, __file__] + HEADERS):
            return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(command(), check=True)
    return OUT


_lib = None


def load():
    global _lib
    if _lib is None:
        lib = C.CDLL(build())
        lib.cpu_port_forward.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Instance_t),
                                         C.c_void_p, C.c_int]
        lib.cpu_port_forward.restype = C.c_int
        lib.cpu_port_forward_many.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(Instance_t),
                                              C.c_int, C.c_void_p, C.c_int]
        lib.cpu_port_forward_many.restype = C.c_int
        lib.cpu_port_max_threads.restype = C.c_int
        _lib = lib
    return _lib


def max_threads():
    return int(load().cpu_port_max_threads())


class Prepared:
    """One synthetic instance (jax-gcm_b200/synthetic.py Instance) with its output arrays and
    argument structs, ready to run repeatedly."""

    def __init__(self, inst, params=None):
        pkg = importlib.import_module("jax-gcm_b200")
        L = pkg._lib
        P = pkg.Parameters.default() if params is None else params
        self.inst = inst
        self.pstruct = P.to_struct()
        vg = L.VGrid()
        vt = pkg.physics.initialize_vertical(inst.kx)
        for name, arr in zip(("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp"), vt[:6]):
            tgt = getattr(vg, name)
            for i, x in enumerate(arr):
                tgt[i] = float(x)
        for k in range(inst.kx):
            vg.wvi[k][0], vg.wvi[k][1] = float(vt[6][k, 0]), float(vt[6][k, 1])
        self.vgrid = vg
        kx, ix, il = inst.kx, inst.ix, inst.il
        self.out = {n: np.zeros((kx, ix, il), np.float32) for n in ("du", "dv", "dt", "dq")}
        for n in ("precnv", "precls", "cloudc", "rsds", "rlds"):
            self.out[n] = np.zeros((ix, il), np.float32)
        for n in ("iptop", "icltop"):
            self.out[n] = np.zeros((ix, il), np.int32)
        self.inputs = {n: np.ascontiguousarray(getattr(inst, n), np.float32) for n in _F}
        flags = (L.SPD_LFLUXLAND if inst.lfluxland else 0)
        if P.surface_flux.lscasym:
            flags |= L.SPD_LSCASYM
        if P.surface_flux.lskineb:
            flags |= L.SPD_LSKINEB
        inc = 1.0 if P.forcing.increase_co2 else 0.0
        ablco2 = np.float32(6.0) * np.exp(np.float32(inc * 0.005) * (
            np.float32(inst.model_year) + np.float32(inst.tyear) -
            np.float32(P.forcing.co2_year_ref)))
        s = Instance_t(kx, ix, il, flags, int(inst.model_step), float(np.float32(inst.tyear)),
                       float(ablco2))
        for n, a in self.inputs.items():
            setattr(s, n, a.ctypes.data)
        for n, a in self.out.items():
            setattr(s, n, a.ctypes.data)
        self.struct = s
        self.rows = np.zeros(il * 6, np.float32)

    def run(self, nthreads=0):
        rc = load().cpu_port_forward(C.byref(self.vgrid), C.byref(self.pstruct),
                                     C.byref(self.struct), self.rows.ctypes.data, nthreads)
        if rc != 0:
            raise RuntimeError(f"cpu_port_forward failed ({rc})")
        o = self.out
        return dict(u_wind=o["du"], v_wind=o["dv"], temperature=o["dt"],
                    specific_humidity=o["dq"], precnv=o["precnv"], precls=o["precls"],
                    cloudc=o["cloudc"], rsds=o["rsds"], rlds=o["rlds"], iptop=o["iptop"],
                    icltop=o["icltop"])


class Batch:
    """Many prepared instances run in one parallel region (cpu_port_forward_many): the
    benchmark's CPU arm over a whole ensemble."""

    def __init__(self, insts, params=None):
        self.items = [Prepared(i, params) for i in insts]
        n = len(self.items)
        pkg = importlib.import_module("jax-gcm_b200")
        self.vgs = (pkg._lib.VGrid * n)(*[p.vgrid for p in self.items])
        self.ps = (pkg._lib.Params * n)(*[p.pstruct for p in self.items])
        self.structs = (Instance_t * n)(*[p.struct for p in self.items])
        self.rows = np.zeros(6 * sum(p.inst.il for p in self.items), np.float32)
        self.columns = sum(p.inst.columns for p in self.items)

    def run(self, nthreads=0):
        rc = load().cpu_port_forward_many(C.byref(self.vgs), C.byref(self.ps), self.structs,
                                          len(self.items), self.rows.ctypes.data, nthreads)
        if rc != 0:
            raise RuntimeError(f"cpu_port_forward_many failed ({rc})")
        return [p.out for p in self.items]
