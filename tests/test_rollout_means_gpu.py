"""One-day rollouts of the column physics: global means against the oracle.

The reference checks 1-day Model runs by global-mean temperature, humidity and precipitation
(within 1e-3 relative).  Without JAX or its dynamical core here, the same check runs on the
physics alone: 48 explicit steps of dt = 1800 s (jax-gcm_b200/rollout.py, the fused physics
step with verify_state/verify_tendencies), once through the CUDA path and once through the
float32 oracle (and the float64 oracle, for the stated x64 distance), from the same seeded
state.  Compared: the area- and sigma-weighted global means of T and q after the day, and the
area-weighted global mean of the day-averaged precipitation (convective plus large-scale).
"""
import importlib
from dataclasses import replace as dc_replace

import numpy as np
import pytest
import torch

from oracle import speedy_oracle as O

pytestmark = pytest.mark.gpu

pkg = importlib.import_module("jax-gcm_b200")
R = pkg.rollout
NSTEPS, DT = 48, 1800.0
REL = 1e-3


def oracle_rollout(inst, dtype):
    st, fo, ge, da, pr = inst.oracle_args(O.default_parameters(dtype))
    st, fo, ge, da, pr = O.cast_inputs(st, fo, ge, da, pr, dtype)
    dt = dtype(DT)
    acc = np.zeros(st.normalized_surface_pressure.shape, dtype)
    for n in range(NSTEPS):
        dn = O.make_date(da.tyear, da.model_year, int(da.model_step) + n, da.dt_seconds, dtype)
        tend, data = O.physics_step(st, fo, ge, dn, pr, time_step=dt, fuse_verify=True)
        acc = acc + data.convection.precnv + data.condensation.precls
        for k in ("u_wind", "v_wind", "temperature", "specific_humidity"):
            setattr(st, k, (getattr(st, k) + dt * getattr(tend, k)).astype(dtype))
    return st.temperature, st.specific_humidity, acc / dtype(NSTEPS)


def global_means(inst, t, q, precip):
    w = np.cos(inst.lat.astype(np.float64))[None, :]
    w = np.broadcast_to(w, (inst.ix, inst.il))
    dhs = O.vertical_tables(inst.kx, np.float64)[2]
    area = lambda a: float((np.asarray(a, np.float64) * w).sum() / w.sum())
    vert = lambda a: area(np.tensordot(dhs, np.asarray(a, np.float64), axes=1) / dhs.sum())
    return {"T": vert(t), "q": vert(q), "precip": area(precip)}


@pytest.mark.parametrize("which", ["t31_aquaplanet", "land_t31_k8", "land_t42_k16"])
def test_one_day_global_means_match_oracle(which):
    syn = pkg.synthetic
    inst = {"t31_aquaplanet": lambda: syn.config0_instance(seed=3, lfluxland=True),
            "land_t31_k8": lambda: syn.land_instance(31, 96, 48, 8),
            "land_t42_k16": lambda: syn.land_instance(42, 128, 64, 16)}[which]()
    st, fo, ge, da = pkg.instance_to_device(inst, "cuda")
    x, pr = R.rollout_with_precipitation(None, st, fo, ge, da, nsteps=NSTEPS, dt=DT)
    gpu = global_means(inst, x.temperature.cpu().numpy(), x.specific_humidity.cpu().numpy(),
                       pr.cpu().numpy())
    o32 = global_means(inst, *oracle_rollout(inst, np.float32))
    o64 = global_means(inst, *oracle_rollout(inst, np.float64))
    rel = {k: abs(gpu[k] - o32[k]) / abs(o32[k]) for k in gpu}
    rel64 = {k: abs(gpu[k] - o64[k]) / abs(o64[k]) for k in gpu}
    print(which, "gpu", gpu, "rel vs oracle32", rel, "rel vs oracle64", rel64)
    assert gpu["precip"] > 0.0  # the day rains: the precipitation check is not vacuous
    assert all(r <= REL for r in rel.values()), rel
    assert all(r <= REL for r in rel64.values()), rel64
