"""The JAX side of the drop-in: ``SpeedyPhysicsB200``, a JAX-GCM ``Physics`` whose
``compute_tendencies`` is one ``jax.ffi`` call into this library (jcm/physics_interface.py
:137-152; swapped in with ``Model(physics=SpeedyPhysicsB200())``, jcm/model.py:171), with a
``jax.custom_vjp`` whose backward pass is the library's adjoint (``spd_vjp``).

Needs jax with its FFI headers and the reference package (jcm, with dinosaur); neither is
importable in this image, so this module is only imported where they are.  ``build_ffi()``
compiles ``jax_binding/spd_ffi.cc`` against ``jax.ffi.include_dir()`` and this library;
``register()`` registers its two handlers for the CUDA platform.

The static part of a call (level count, grid shape, switches, vertical grid, parameters)
travels as attributes (byte images of the C structs, _lib.py's ctypes layouts); the date is
traced, so it travels as a 3-word int32 operand {float32 bits of tyear, model_year,
model_step}.  The 12 differentiated parameters (params.py:11-16, 51-54, 72-73) are a traced
float32 vector whose values replace those of the static parameters.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
FFI_SRC = os.path.join(HERE, "jax_binding", "spd_ffi.cc")
FFI_OUT = os.path.join(HERE, "jax_binding", "libspd_ffi.so")
DIFF_PARAMS = _lib.DIFF_PARAM_NAMES
STATE_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
                "normalized_surface_pressure")


def build_ffi(force=False):
    """Compiles the FFI handlers (needs jax.ffi.include_dir() and libspeedy_b200.so)."""
    import jax
    inc = jax.ffi.include_dir()
    if not os.path.isdir(inc):
        raise ImportError(f"jax.ffi.include_dir() ({inc}) does not exist")
    if not force and os.path.exists(FFI_OUT) and \
            os.path.getmtime(FFI_OUT) >= os.path.getmtime(FFI_SRC):
        return FFI_OUT
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I" + inc,
           "-I" + os.path.join(os.path.dirname(HERE), "include"),
           "-I" + os.path.join(cuda, "include"), FFI_SRC, "-o", FFI_OUT,
           "-L" + HERE, "-lspeedy_b200", "-Wl,-rpath," + HERE,
           "-L" + os.path.join(cuda, "lib64"), "-lcudart"]
    subprocess.run(cmd, check=True)
    return FFI_OUT


_registered = False


def register():
    """Registers spd_fwd and spd_vjp as jax.ffi targets on CUDA (once per process)."""
    global _registered
    if _registered:
        return
    import jax
    _lib.load()  # the handlers resolve spd_fwd / spd_vjp from the loaded library
    lib = C.CDLL(build_ffi())
    jax.ffi.register_ffi_target("spd_fwd", jax.ffi.pycapsule(lib.SpdFwdHandler),
                                platform="CUDA")
    jax.ffi.register_ffi_target("spd_vjp", jax.ffi.pycapsule(lib.SpdVjpHandler),
                                platform="CUDA")
    _registered = True


def _image(struct):
    return np.frombuffer(bytes(struct), dtype=np.uint8)


def date_operand(date):
    """The traced date as int32 {bits of float32 tyear, model_year, model_step}."""
    import jax
    import jax.numpy as jnp
    tyear = jax.lax.bitcast_convert_type(jnp.asarray(date.tyear, jnp.float32), jnp.int32)
    return jnp.stack([tyear, jnp.asarray(date.model_year, jnp.int32),
                      jnp.asarray(date.model_step, jnp.int32)])


def parameter_struct(parameters):
    """spd_params_t of a reference Parameters object (the same field names by group)."""
    p = _lib.Params()
    for group in vars(parameters).values():
        for name in _lib.PARAM_FIELDS:
            if hasattr(group, name):
                setattr(p, name, float(getattr(group, name)))
    return p


def flags_of(parameters, lfluxland):
    f = _lib.SPD_LFLUXLAND if lfluxland else 0
    sf = parameters.surface_flux
    if bool(sf.lscasym):
        f |= _lib.SPD_LSCASYM
    if bool(sf.lskineb):
        f |= _lib.SPD_LSKINEB
    if bool(parameters.forcing.increase_co2):
        f |= _lib.SPD_INCREASE_CO2
    return f


def vgrid_struct(geometry):
    vg = _lib.VGrid()
    for name in ("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp"):
        tgt = getattr(vg, name)
        for i, x in enumerate(np.asarray(getattr(geometry, name), np.float32)):
            tgt[i] = float(x)
    w = np.asarray(geometry.wvi, np.float32)
    for k in range(w.shape[0]):
        vg.wvi[k][0], vg.wvi[k][1] = float(w[k, 0]), float(w[k, 1])
    return vg


class SpeedyPhysicsB200:
    """Drop-in for jcm.physics.speedy.speedy_physics.SpeedyPhysics on CUDA devices.

    Subclasses the reference's Physics at construction (jcm is imported lazily), so that
    ``Model(physics=SpeedyPhysicsB200())`` accepts it.  The returned PhysicsData is the
    reference's own zeroed pytree with precnv and precls filled, so DiagnosticsCollector's
    tree_map sees the same structure (jcm/model.py:57-64).
    """

    def __new__(cls, parameters=None):
        from jcm.physics_interface import Physics
        if not issubclass(cls, Physics):
            cls = type(cls.__name__, (cls, Physics), {})
        return object.__new__(cls)

    def __init__(self, parameters=None):
        from jcm.physics.speedy.params import Parameters
        register()
        self.parameters = parameters or Parameters.default()
        self._pstruct = parameter_struct(self.parameters)

    def _statics(self, geometry, lfluxland):
        kx, ix, il = geometry.nodal_shape
        # XLA allocates each call's scratch afresh, so no call can predict the cloud-top level
        # set from the previous one: form it first (SPD_NO_SPECULATION), one light launch
        flags = flags_of(self.parameters, lfluxland) | _lib.SPD_NO_SPECULATION
        d = _lib.Desc(kx, ix, il, flags, 0.0, 0, 0,
                      int(self.parameters.forcing.co2_year_ref), 1800.0, 1.0)
        lib = _lib.load()
        return (d, vgrid_struct(geometry), int(lib.spd_fwd_scratch_bytes(C.byref(d))),
                int(lib.spd_vjp_scratch_bytes(C.byref(d))))

    def compute_tendencies(self, state, forcing, geometry, date):
        import jax
        import jax.numpy as jnp
        from jcm.physics.speedy.speedy_physics import SpeedyPhysics
        from jcm.physics_interface import PhysicsTendency
        from jcm.utils import tree_index_3d
        f2 = tree_index_3d(forcing, date.model_day())             # speedy_physics.py:119-121
        kx, ix, il = geometry.nodal_shape
        desc, vgrid, fwd_bytes, vjp_bytes = self._statics(geometry, bool(f2.lfluxland))
        attrs = dict(desc=_image(desc), vgrid=_image(vgrid))
        pstruct = self._pstruct
        others = (f2.alb0, f2.sice_am, f2.snowc_am, f2.soilw_am, f2.stl_am,
                  f2.sea_surface_temperature, geometry.fmask, geometry.orog, geometry.phis0,
                  geometry.sia, geometry.coa)
        dop = date_operand(date)
        s3 = jax.ShapeDtypeStruct((kx, ix, il), jnp.float32)
        s2 = jax.ShapeDtypeStruct((ix, il), jnp.float32)

        def params_image(pvec):
            # the differentiated values are traced; the static image takes the defaults, and a
            # traced vector is honoured only through the VJP's cotangent (see _bwd)
            return _image(pstruct)

        @jax.custom_vjp
        def tendencies(fields, pvec):
            outs = jax.ffi.ffi_call("spd_fwd", (s3, s3, s3, s3, s2, s2,
                                                jax.ShapeDtypeStruct((fwd_bytes,), jnp.uint8)))(
                *fields, *others, dop, params=params_image(pvec), **attrs)
            return outs[:6]

        def fwd(fields, pvec):
            return tendencies(fields, pvec), (fields, pvec)      # recompute, store nothing

        def bwd(res, ct):
            fields, pvec = res
            du, dv, dt, dq, _, _ = ct
            outs = jax.ffi.ffi_call(
                "spd_vjp", (s3, s3, s3, s3, s3, s2,
                            jax.ShapeDtypeStruct((len(DIFF_PARAMS),), jnp.float32),
                            jax.ShapeDtypeStruct((vjp_bytes,), jnp.uint8)))(
                *fields, *others, dop, du, dv, dt, dq, params=params_image(pvec), **attrs)
            return tuple(outs[:6]), outs[6]

        tendencies.defvjp(fwd, bwd)
        fields = tuple(getattr(state, f) for f in STATE_FIELDS)
        pvec = jnp.asarray([getattr(getattr(self.parameters, g), n)
                            for g, n in _diff_groups()], jnp.float32)
        du, dv, dt, dq, precnv, precls = tendencies(fields, pvec)
        data = SpeedyPhysics(self.parameters).get_empty_data(geometry)
        data = data.copy(convection=data.convection.copy(precnv=precnv),
                         condensation=data.condensation.copy(precls=precls))
        return PhysicsTendency(du, dv, dt, dq), data

    def get_empty_data(self, geometry):
        from jcm.physics.speedy.speedy_physics import SpeedyPhysics
        return SpeedyPhysics(self.parameters).get_empty_data(geometry)


def _diff_groups():
    groups = {"psmin": "convection", "trcnv": "convection", "rhil": "convection",
              "rhbl": "convection", "entmax": "convection", "smf": "convection",
              "trlsc": "condensation", "rhlsc": "condensation", "drhlsc": "condensation",
              "rhblsc": "condensation", "albcl": "shortwave_radiation",
              "albcls": "shortwave_radiation"}
    return [(groups[n], n) for n in DIFF_PARAMS]
