"""Adjoint of the SPEEDY column physics and its autograd bindings.

``vjp`` is the counterpart of ``jax.vjp`` applied to ``SpeedyPhysics.compute_tendencies``
(jcm/physics/speedy/speedy_physics.py:88-127) for the tendency outputs: given cotangents of the
four tendency planes it returns the gradients with respect to the PhysicsState planes and to
the 12 tuning parameters (params.py:11-16, :51-54, :72-73).  It runs ``spd_vjp``, which
recomputes each column's forward on a per-thread tape instead of storing the forward.

``speedy_b200::tendencies`` is the same forward as a ``torch.library`` custom op whose autograd
rule is ``spd_vjp``; ``SpeedyTendencies`` wraps it for PhysicsState inputs.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from .physics import (Parameters, PhysicsState, PhysicsTendency, SpeedyPhysics,
                      current_raw_stream)

DIFF_PARAMS = [("convection", "psmin"), ("convection", "trcnv"), ("convection", "rhil"),
               ("convection", "rhbl"), ("convection", "entmax"), ("convection", "smf"),
               ("condensation", "trlsc"), ("condensation", "rhlsc"),
               ("condensation", "drhlsc"), ("condensation", "rhblsc"),
               ("shortwave_radiation", "albcl"), ("shortwave_radiation", "albcls")]

_SCRATCH = {}


def _scratch(nbytes, device):
    key = (str(device),)
    buf = _SCRATCH.get(key)
    if buf is None or buf.numel() < nbytes:
        buf = torch.empty(nbytes, dtype=torch.uint8, device=device)
        _SCRATCH[key] = buf
    return buf


def _input_struct(state, forcing, geometry):
    f2 = forcing
    t = dict(u_wind=state.u_wind, v_wind=state.v_wind, temperature=state.temperature,
             specific_humidity=state.specific_humidity, geopotential=state.geopotential,
             normalized_surface_pressure=state.normalized_surface_pressure, alb0=f2.alb0,
             sice_am=f2.sice_am, snowc_am=f2.snowc_am, soilw_am=f2.soilw_am, stl_am=f2.stl_am,
             sea_surface_temperature=f2.sea_surface_temperature, fmask=geometry.fmask,
             orog=geometry.orog, phis0=geometry.phis0, sia=geometry.sia, coa=geometry.coa)
    dev = state.temperature.device
    didx = state.temperature.get_device()
    ptrs = []
    for k in _lib.INPUT_FIELDS:
        v = t[k]
        if v.dtype is not torch.float32 or not v.is_contiguous() or v.get_device() != didx:
            v = t[k] = v.to(device=dev, dtype=torch.float32).contiguous()
        ptrs.append(v.data_ptr())
    return _lib.Inputs(*ptrs), t


def vjp(physics: SpeedyPhysics, state: PhysicsState, forcing, geometry, date,
        cotangent: PhysicsTendency):
    """(PhysicsState of gradients, tensor[12] of parameter gradients) for the cotangent."""
    lib = _lib.load()
    dev = state.temperature.device
    _lib.preload(dev.index if dev.index is not None else torch.cuda.current_device())
    f2 = forcing.day_slice(date.model_day())
    inp, keep = _input_struct(state, f2, geometry)
    ct = {k: getattr(cotangent, k).to(device=dev, dtype=torch.float32).contiguous()
          for k in ("u_wind", "v_wind", "temperature", "specific_humidity")}
    cts = _lib.Cotangents(**{k: v.data_ptr() for k, v in ct.items()})
    e = lambda ref: torch.empty_like(ref)
    g = dict(u_wind=e(state.u_wind), v_wind=e(state.v_wind), temperature=e(state.temperature),
             specific_humidity=e(state.specific_humidity), geopotential=e(state.geopotential),
             normalized_surface_pressure=e(state.normalized_surface_pressure),
             params=torch.empty(12, dtype=torch.float32, device=dev))
    grads = _lib.Grads(**{k: v.data_ptr() for k, v in g.items()})
    desc = physics.desc(geometry, date, forcing.lfluxland)
    n = lib.spd_vjp_scratch_bytes(C.byref(desc))
    sc = _scratch(n, dev)
    stream = current_raw_stream(state.temperature.get_device())
    rc = lib.spd_vjp(C.byref(desc), C.byref(geometry.vgrid()), C.byref(physics._pstruct),
                     C.byref(inp), C.byref(cts), C.byref(grads), C.c_void_p(sc.data_ptr()), n,
                     C.c_void_p(stream))
    _lib.check(rc, "spd_vjp")
    gs = PhysicsState(g["u_wind"], g["v_wind"], g["temperature"], g["specific_humidity"],
                      g["geopotential"], g["normalized_surface_pressure"])
    return gs, g["params"]


# ---------------------------------------------------------------------------------------------
# torch.library op + autograd
# ---------------------------------------------------------------------------------------------
class _Ctx:
    """The non-tensor arguments of one op call (kept on the Python side)."""
    registry = {}
    counter = 0


def _register(physics, forcing, geometry, date):
    _Ctx.counter += 1
    _Ctx.registry[_Ctx.counter] = (physics, forcing, geometry, date)
    if len(_Ctx.registry) > 64:
        _Ctx.registry.pop(next(iter(_Ctx.registry)))
    return _Ctx.counter


@torch.library.custom_op("speedy_b200::tendencies", mutates_args=())
def _tendencies_op(u: torch.Tensor, v: torch.Tensor, t: torch.Tensor, q: torch.Tensor,
                   phi: torch.Tensor, psa: torch.Tensor, params: torch.Tensor,
                   handle: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
    physics, forcing, geometry, date = _Ctx.registry[handle]
    phys = physics
    if params is not None and params.numel() == 12:
        vals = params.detach().cpu().numpy().astype(np.float64)
        kw = {f"{g}__{n}": float(x) for (g, n), x in zip(DIFF_PARAMS, vals)}
        phys = SpeedyPhysics(physics.parameters.with_values(**kw), fuse_verify=physics.fuse_verify,
                             time_step=physics.time_step, q_tend_scale=physics.q_tend_scale,
                             diagnostics=False,
                             orographic_correction=physics.orographic_correction)
    st = PhysicsState(u.contiguous(), v.contiguous(), t.contiguous(), q.contiguous(),
                      phi.contiguous(), psa.contiguous())
    tend, _ = phys.compute_tendencies(st, forcing, geometry, date)
    return tend.u_wind, tend.v_wind, tend.temperature, tend.specific_humidity


@_tendencies_op.register_fake
def _(u, v, t, q, phi, psa, params, handle):
    return torch.empty_like(u), torch.empty_like(v), torch.empty_like(t), torch.empty_like(q)


def _setup_context(ctx, inputs, output):
    u, v, t, q, phi, psa, params, handle = inputs
    ctx.save_for_backward(u, v, t, q, phi, psa, params)
    ctx.handle = handle


def _backward(ctx, gu, gv, gt, gq):
    u, v, t, q, phi, psa, params = ctx.saved_tensors
    physics, forcing, geometry, date = _Ctx.registry[ctx.handle]
    phys = physics
    if params is not None and params.numel() == 12:
        vals = params.detach().cpu().numpy().astype(np.float64)
        kw = {f"{g}__{n}": float(x) for (g, n), x in zip(DIFF_PARAMS, vals)}
        phys = SpeedyPhysics(physics.parameters.with_values(**kw), fuse_verify=physics.fuse_verify,
                             time_step=physics.time_step, q_tend_scale=physics.q_tend_scale,
                             diagnostics=False,
                             orographic_correction=physics.orographic_correction)
    z = lambda ref: torch.zeros_like(ref)
    cot = PhysicsTendency(gu if gu is not None else z(u), gv if gv is not None else z(v),
                          gt if gt is not None else z(t), gq if gq is not None else z(q))
    gs, gp = vjp(phys, PhysicsState(u, v, t, q, phi, psa), forcing, geometry, date, cot)
    return (gs.u_wind, gs.v_wind, gs.temperature, gs.specific_humidity, gs.geopotential,
            gs.normalized_surface_pressure, gp.to(params.device) if params is not None else None,
            None)


_tendencies_op.register_autograd(_backward, setup_context=_setup_context)


def parameter_vector(parameters: Optional[Parameters] = None, device="cpu"):
    """The 12 differentiated parameters as a float32 tensor (order of DIFF_PARAMS)."""
    p = parameters or Parameters.default()
    return torch.tensor([getattr(getattr(p, g), n) for g, n in DIFF_PARAMS], dtype=torch.float32,
                        device=device)


def tendencies(physics: SpeedyPhysics, state: PhysicsState, forcing, geometry, date,
               params: Optional[torch.Tensor] = None):
    """Differentiable tendencies: a PhysicsTendency whose planes carry autograd back to the
    state tensors and to ``params`` (a 12-vector, see parameter_vector)."""
    if params is None:
        params = parameter_vector(physics.parameters)
    h = _register(physics, forcing, geometry, date)
    du, dv, dt, dq = _tendencies_op(state.u_wind, state.v_wind, state.temperature,
                                    state.specific_humidity, state.geopotential,
                                    state.normalized_surface_pressure, params, h)
    return PhysicsTendency(du, dv, dt, dq)
