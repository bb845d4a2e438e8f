"""ctypes binding of ``libspeedy_b200.so`` (declared in ``include/speedy_b200.h``).

The library is built in-tree (``build.py``) and loaded on first use.  There is no fallback:
if the shared library is missing or cannot be loaded, every compute entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
# SPEEDY_B200_LIB names another build of the library (e.g. a profiling variant).
LIB_PATH = os.environ.get("SPEEDY_B200_LIB") or os.path.join(HERE, "libspeedy_b200.so")
MAX_KX = 16

SPD_LFLUXLAND = 1 << 0
SPD_LSCASYM = 1 << 1
SPD_LSKINEB = 1 << 2
SPD_INCREASE_CO2 = 1 << 3
SPD_FUSE_VERIFY = 1 << 4
SPD_OROGRAPHIC = 1 << 5
SPD_ACCUMULATE_DIAGNOSTICS = 1 << 6
SPD_LOW_LEVEL_WINDS = 1 << 7
SPD_NO_SPECULATION = 1 << 8


class Desc(C.Structure):
    _fields_ = [("kx", C.c_int32), ("ix", C.c_int32), ("il", C.c_int32), ("flags", C.c_uint32),
                ("tyear", C.c_float), ("model_year", C.c_int32), ("model_step", C.c_int32),
                ("co2_year_ref", C.c_int32), ("dt_seconds", C.c_float),
                ("q_tend_scale", C.c_float)]


class VGrid(C.Structure):
    _fields_ = [("hsg", C.c_float * (MAX_KX + 1)), ("fsg", C.c_float * MAX_KX),
                ("dhs", C.c_float * MAX_KX), ("sigl", C.c_float * MAX_KX),
                ("grdsig", C.c_float * MAX_KX), ("grdscp", C.c_float * MAX_KX),
                ("wvi", (C.c_float * 2) * MAX_KX)]


PARAM_FIELDS = [
    "psmin", "trcnv", "rhil", "rhbl", "entmax", "smf",
    "trlsc", "rhlsc", "drhlsc", "rhblsc",
    "albcl", "albcls", "absdry", "absaer", "abswv1", "abswv2", "abscl1", "abscl2",
    "ablwin", "ablwv1", "ablwv2", "ablcl1", "ablcl2",
    "rhcl1", "rhcl2", "qacl", "wpcl", "pmaxcl", "clsmax", "clsminl", "gse_s0", "gse_s1",
    "albsea", "albice", "albsn", "epslw", "emisfc",
    "fwind0", "ftemp0", "fhum0", "cdl", "cds", "chl", "chs", "vgust", "ctday", "dtheta", "fstab",
    "clambda", "clambsn", "hdrag",
    "trshc", "trvdi", "trvds", "redshc", "rhgrad", "segrad",
]


class Params(C.Structure):
    _fields_ = [(n, C.c_float) for n in PARAM_FIELDS]


INPUT_FIELDS = ["u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
                "normalized_surface_pressure", "alb0", "sice_am", "snowc_am", "soilw_am",
                "stl_am", "sea_surface_temperature", "fmask", "orog", "phis0", "sia", "coa"]
OUTPUT_FIELDS = ["u_wind", "v_wind", "temperature", "specific_humidity", "precnv", "precls",
                 "cbmf", "cloudc", "cloudstr", "rsds", "rsns", "ftop_sw", "rlds", "rlns",
                 "ftop_lw", "tsfc", "tskin", "shf", "evap", "iptop", "icltop"]


class Inputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in INPUT_FIELDS]


class Outputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in OUTPUT_FIELDS]


class Class(C.Structure):
    _fields_ = [("desc", Desc), ("vgrid", VGrid), ("params", Params)]


class Member(C.Structure):
    _fields_ = [("inp", Inputs), ("out", Outputs), ("ix", C.c_int32), ("il", C.c_int32),
                ("cls", C.c_int32), ("reserved", C.c_int32)]


class PlanInfo(C.Structure):
    _fields_ = [("nmembers", C.c_int32), ("ntiles", C.c_int32),
                ("levelset_offset", C.c_uint64), ("levelset_bytes", C.c_uint64),
                ("plan_bytes", C.c_uint64)]


MAX_CLASSES = 4


class Cotangents(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("u_wind", "v_wind", "temperature", "specific_humidity")]


class Grads(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("u_wind", "v_wind", "temperature", "specific_humidity",
                                          "geopotential", "normalized_surface_pressure",
                                          "params")]


class VjpMember(C.Structure):
    _fields_ = [("inp", Inputs), ("ct", Cotangents), ("grads", Grads), ("ix", C.c_int32),
                ("il", C.c_int32), ("cls", C.c_int32), ("reserved", C.c_int32)]


DIFF_PARAM_NAMES = ["psmin", "trcnv", "rhil", "rhbl", "entmax", "smf", "trlsc", "rhlsc",
                    "drhlsc", "rhblsc", "albcl", "albcls"]

STATUS = {0: "ok", 1: "null pointer", 2: "bad shape", 3: "unsupported kx", 4: "bad scratch",
          5: "CUDA error", 7: "misaligned pointer",
          8: "il above the no-allocation entry point's limit",
          9: "an output field overlaps an input or another output",
          10: "the stream belongs to another device than the current one"}
NOALLOC_MAX_IL = 2048
GRID_PER_TILE = -1  # SPD_GRID_PER_TILE

_lib = None
_lock = threading.Lock()


class SpeedyLibraryError(RuntimeError):
    pass


class HsDesc(C.Structure):
    _fields_ = [("kx", C.c_int32), ("ix", C.c_int32), ("il", C.c_int32), ("reserved", C.c_int32),
                ("sigma_b", C.c_float), ("kf", C.c_float), ("ka", C.c_float), ("ks", C.c_float),
                ("min_t", C.c_float), ("max_t", C.c_float), ("dt_y", C.c_float),
                ("dthz", C.c_float), ("kappa", C.c_float), ("sigma", C.c_float * 16)]


def _declare(lib):
    P = C.POINTER
    lib.spd_fwd_scratch_bytes.argtypes = [P(Desc)]
    lib.spd_fwd_scratch_bytes.restype = C.c_size_t
    lib.spd_fwd.argtypes = [P(Desc), P(VGrid), P(Params), P(Inputs), P(Outputs), C.c_void_p,
                            C.c_size_t, C.c_void_p]
    lib.spd_fwd.restype = C.c_int
    lib.spd_fwd_marked.argtypes = lib.spd_fwd.argtypes + [C.c_void_p]
    lib.spd_fwd_marked.restype = C.c_int
    lib.spd_status_string.argtypes = [C.c_int]
    lib.spd_status_string.restype = C.c_char_p
    lib.spd_abi_version.argtypes = []
    lib.spd_abi_version.restype = C.c_int
    lib.spd_default_params.argtypes = [P(Params)]
    lib.spd_default_params.restype = None
    lib.spd_fwd_noalloc.argtypes = [P(Desc), P(VGrid), P(Params), P(Inputs), P(Outputs),
                                    C.c_void_p]
    lib.spd_fwd_noalloc.restype = C.c_int
    lib.spd_ensemble_plan_bytes.argtypes = [P(Member), C.c_int]
    lib.spd_ensemble_plan_bytes.restype = C.c_size_t
    lib.spd_ensemble_plan.argtypes = [P(Class), C.c_int, P(Member), C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_size_t, P(PlanInfo)]
    lib.spd_ensemble_plan.restype = C.c_int
    lib.spd_ensemble_fwd.argtypes = [P(Class), C.c_int, C.c_void_p, P(PlanInfo), C.c_int,
                                     C.c_void_p]
    lib.spd_ensemble_fwd.restype = C.c_int
    lib.spd_ensemble_fwd_marked.argtypes = lib.spd_ensemble_fwd.argtypes + [C.c_void_p]
    lib.spd_ensemble_fwd_marked.restype = C.c_int
    lib.spd_vjp_scratch_bytes.argtypes = [P(Desc)]
    lib.spd_vjp_scratch_bytes.restype = C.c_size_t
    lib.spd_vjp.argtypes = [P(Desc), P(VGrid), P(Params), P(Inputs), P(Cotangents), P(Grads),
                            C.c_void_p, C.c_size_t, C.c_void_p]
    lib.spd_vjp.restype = C.c_int
    lib.spd_preload.argtypes = []
    lib.spd_preload.restype = C.c_int
    lib.spd_selftest_packed.argtypes = [C.c_int, C.c_uint32, P(C.c_uint)]
    lib.spd_selftest_packed.restype = C.c_int
    lib.spd_ensemble_vjp_plan_bytes.argtypes = [P(VjpMember), C.c_int]
    lib.spd_ensemble_vjp_plan_bytes.restype = C.c_size_t
    lib.spd_ensemble_vjp_plan.argtypes = [P(Class), C.c_int, P(VjpMember), C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_size_t, P(PlanInfo)]
    lib.spd_ensemble_vjp_plan.restype = C.c_int
    lib.spd_ensemble_vjp.argtypes = [P(Class), C.c_int, C.c_void_p, P(PlanInfo), C.c_int,
                                     C.c_void_p]
    lib.spd_ensemble_vjp.restype = C.c_int
    lib.spd_held_suarez.argtypes = [P(HsDesc)] + [C.c_void_p] * 10
    lib.spd_held_suarez.restype = C.c_int
    for name, spec in EXTRA_DECLS.items():
        fn = getattr(lib, name, None)
        if fn is not None:
            fn.argtypes, fn.restype = spec(P)


EXTRA_DECLS = {}


def load():
    """Loads the CUDA library (once).  Raises SpeedyLibraryError when it is missing."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise SpeedyLibraryError(
                    f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                    "g.build()'` (nvcc, sm_100a); there is no CPU fallback")
            try:
                lib = C.CDLL(LIB_PATH)
            except OSError as e:
                raise SpeedyLibraryError(f"cannot load {LIB_PATH}: {e}") from e
            _declare(lib)
            _lib = lib
    return _lib


def check(rc, what="spd call"):
    if rc != 0:
        msg = load().spd_status_string(rc).decode()
        raise SpeedyLibraryError(f"{what} failed with status {rc}: {msg}")


_preloaded = set()


def preload(device_index: int):
    """Loads every kernel on ``device_index`` once per process (spd_preload), so that lazy
    module loading never waits on running kernels at a first launch."""
    if device_index in _preloaded:
        return
    import torch
    lib = load()
    with torch.cuda.device(device_index):
        check(lib.spd_preload(), "spd_preload")
    _preloaded.add(device_index)
