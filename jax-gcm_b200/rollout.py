"""Explicit column rollouts and their adjoint with recompute checkpoints.

A column rollout advances the PhysicsState with the physics alone (no dynamics): each step
applies the fused physics step of ``get_physical_tendencies`` (verify_state, the SPEEDY
physics, verify_tendencies; jcm/physics_interface.py:305-376) and an explicit Euler update

    x_{n+1} = x_n + dt * f_n(x_n),   x = (u, v, T, q),

with geopotential and surface pressure held fixed and the model step advancing (the shortwave
runs on every third step, speedy_physics.py:108-113).

``rollout_vjp`` returns the gradient of <cotangent, x_N> with respect to x_0, the fixed
geopotential and surface pressure, and the 12 tuning parameters.  The forward keeps only every
``checkpoint_every``-th state; the reverse recomputes each segment from its checkpoint and runs
the column adjoint (``spd_vjp``) on every step of it, last to first:

    xbar_n = xbar_{n+1} + J_n^T (dt xbar_{n+1}).

The reference differentiates a Model run with jax.checkpoint around the physics terms
(speedy_physics.py:82-86); the segment recompute here is the same trade of memory for work at
the granularity of whole steps.
"""
from __future__ import annotations

from dataclasses import replace
from typing import Optional

import torch

from .adjoint import vjp
from .physics import PhysicsState, PhysicsTendency, SpeedyPhysics

EVOLVED = ("u_wind", "v_wind", "temperature", "specific_humidity")


def _physics(physics: Optional[SpeedyPhysics], dt: float) -> SpeedyPhysics:
    p = physics.parameters if physics is not None else None
    oro = physics.orographic_correction if physics is not None else False
    return SpeedyPhysics(p, fuse_verify=True, time_step=dt, diagnostics=False,
                         orographic_correction=oro)


def _date(date, n):
    return replace(date, model_step=int(date.model_step) + n)


def step(physics: SpeedyPhysics, state: PhysicsState, forcing, geometry, date, dt: float):
    """One explicit step of the fused physics: a new PhysicsState (the four Euler updates in
    one multi-tensor launch)."""
    tend, _ = physics.compute_tendencies(state, forcing, geometry, date)
    u, v, t, q = torch._foreach_add([getattr(state, k) for k in EVOLVED],
                                    [getattr(tend, k) for k in EVOLVED], alpha=dt)
    return PhysicsState(u, v, t, q, state.geopotential, state.normalized_surface_pressure)


def rollout(physics, state, forcing, geometry, date, nsteps=48, dt=1800.0):
    """The state after ``nsteps`` explicit steps of ``dt`` seconds."""
    ph = _physics(physics, dt)
    x = state
    for n in range(nsteps):
        x = step(ph, x, forcing, geometry, _date(date, n), dt)
    return x


def rollout_with_precipitation(physics, state, forcing, geometry, date, nsteps=48,
                               dt=1800.0):
    """``rollout`` that also returns, per column, the precipitation (convective plus
    large-scale, as PhysicsData reports them) averaged over the steps."""
    ph = _physics(physics, dt)
    x = state
    acc = torch.zeros_like(state.normalized_surface_pressure)
    for n in range(nsteps):
        tend, data = ph.compute_tendencies(x, forcing, geometry, _date(date, n))
        acc += data.convection.precnv + data.condensation.precls
        new = {k: getattr(x, k) + dt * getattr(tend, k) for k in EVOLVED}
        x = PhysicsState(new["u_wind"], new["v_wind"], new["temperature"],
                         new["specific_humidity"], x.geopotential, x.normalized_surface_pressure)
    return x, acc / nsteps


def checkpointed_reverse(step_fn, step_vjp_fn, x0, xbar_final, nsteps, checkpoint_every):
    """Reverse pass of x_{n+1} = step_fn(x_n, n) with checkpoints.

    The forward keeps x_0 and every ``checkpoint_every``-th state; the reverse recomputes each
    segment from its checkpoint and applies ``step_vjp_fn(x_n, n, xbar_{n+1}) -> xbar_n`` from
    the last step to the first.  Returns (x_N, xbar_0, peak number of states held)."""
    if checkpoint_every < 1:
        raise ValueError("checkpoint_every must be >= 1")
    ckpt = {0: x0}
    x = x0
    for n in range(nsteps):
        x = step_fn(x, n)
        if (n + 1) % checkpoint_every == 0 and n + 1 < nsteps:
            ckpt[n + 1] = x
    final = x
    held = len(ckpt)
    xb = xbar_final
    for s0 in reversed(range(0, nsteps, checkpoint_every)):
        s1 = min(s0 + checkpoint_every, nsteps)
        xs = [ckpt[s0]]
        for n in range(s0, s1 - 1):
            xs.append(step_fn(xs[-1], n))
        held = max(held, len(ckpt) + len(xs) - 1)
        for n in reversed(range(s0, s1)):
            xb = step_vjp_fn(xs[n - s0], n, xb)
    return final, xb, held


def rollout_vjp(physics, state, forcing, geometry, date, cotangent, nsteps=48, dt=1800.0,
                checkpoint_every=8):
    """(final state, PhysicsState of gradients with respect to the initial state, tensor[12] of
    parameter gradients) for <cotangent, x_N>; ``cotangent`` is a PhysicsTendency-like object
    with u_wind, v_wind, temperature and specific_humidity planes."""
    ph = _physics(physics, dt)
    phi_b = torch.zeros_like(state.geopotential)
    psa_b = torch.zeros_like(state.normalized_surface_pressure)
    par_b = torch.zeros(12, dtype=torch.float32, device=state.temperature.device)

    def fwd(x, n):
        return step(ph, x, forcing, geometry, _date(date, n), dt)

    def rev(x, n, xb):
        ct = PhysicsTendency(*torch._foreach_mul([xb[k] for k in EVOLVED], dt))
        g, gp = vjp(ph, x, forcing, geometry, _date(date, n), ct)
        # the fixed fields' and the parameters' gradients accumulate in place, in one launch
        torch._foreach_add_([phi_b, psa_b, par_b], [g.geopotential, g.normalized_surface_pressure,
                                                   gp])
        return dict(zip(EVOLVED, torch._foreach_add([xb[k] for k in EVOLVED],
                                                    [getattr(g, k) for k in EVOLVED])))

    xb0 = {k: getattr(cotangent, k).to(torch.float32).clone() for k in EVOLVED}
    final, xb, _ = checkpointed_reverse(fwd, rev, state, xb0, nsteps, checkpoint_every)
    grads = PhysicsState(xb["u_wind"], xb["v_wind"], xb["temperature"], xb["specific_humidity"],
                         phi_b, psa_b)
    return final, grads, par_b
