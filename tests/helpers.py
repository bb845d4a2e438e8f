"""Shared helpers of the parity tests: run an Instance through the CUDA path (via the C ABI)
and compare with the oracle under the stated tolerance."""
from __future__ import annotations

import numpy as np

# Parity bar: |cuda - oracle| <= RTOL * max(|oracle|, FLOOR_FRAC * max|oracle field|)
RTOL = 1e-5
FLOOR_FRAC = 1e-3


def to_device(pkg, inst, device="cuda"):
    import torch
    dev = torch.device(device)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    state = pkg.PhysicsState(t(inst.u), t(inst.v), t(inst.t), t(inst.q), t(inst.phi), t(inst.psa))
    forcing = pkg.ForcingData(t(inst.alb0), t(inst.sice), t(inst.snowc), t(inst.soilw),
                              t(inst.stl), t(inst.sst), lfluxland=inst.lfluxland)
    geom = pkg.Geometry.from_grid_shape((inst.ix, inst.il), inst.kx, orography=inst.orog,
                                        fmask=inst.fmask, phis0=inst.phis0, latitudes=inst.lat,
                                        device=dev)
    geom.sia, geom.coa = t(inst.sia), t(inst.coa)
    date = pkg.DateData(inst.tyear, inst.model_year, inst.model_step, inst.dt_seconds)
    return state, forcing, geom, date


def run_gpu_instance(pkg, inst, device="cuda", params=None, **kw):
    import torch
    state, forcing, geom, date = to_device(pkg, inst, device)
    phys = pkg.SpeedyPhysics(params, **kw)
    tend, data = phys.compute_tendencies(state, forcing, geom, date)
    torch.cuda.synchronize()
    c = lambda x: x.detach().cpu().numpy()
    return dict(u_wind=c(tend.u_wind), v_wind=c(tend.v_wind), temperature=c(tend.temperature),
                specific_humidity=c(tend.specific_humidity), precnv=c(data.convection.precnv),
                precls=c(data.condensation.precls), cloudc=c(data.shortwave_rad.cloudc),
                rsds=c(data.shortwave_rad.rsds), rlds=c(data.surface_flux.rlds),
                icltop=c(data.shortwave_rad.icltop), iptop=c(data.convection.iptop))


def oracle_fields(tend, data):
    return dict(u_wind=tend.u_wind, v_wind=tend.v_wind, temperature=tend.temperature,
                specific_humidity=tend.specific_humidity, precnv=data.convection.precnv,
                precls=data.condensation.precls, cloudc=data.shortwave_rad.cloudc,
                rsds=data.shortwave_rad.rsds, rlds=data.surface_flux.rlds,
                icltop=data.shortwave_rad.icltop, iptop=data.convection.iptop)


def column_mask(bad, shape2d):
    """Reduce a per-element failure mask to a per-column mask."""
    b = np.asarray(bad)
    while b.ndim > len(shape2d):
        b = b.any(axis=0)
    return b


def compare_fields(got, tend, data, rtol=RTOL, floor_frac=FLOOR_FRAC):
    ref = oracle_fields(tend, data)
    rep = {}
    for k, r in ref.items():
        if k not in got:
            continue
        g = np.asarray(got[k], np.float64)
        r = np.asarray(r, np.float64)
        if k in ("icltop", "iptop"):
            bad = g != r
            rep[k] = dict(n=r.size, nbad=int(bad.sum()), max_rel=float(bad.mean()), bad=bad)
            continue
        floor = floor_frac * max(np.max(np.abs(r)), 1e-30)
        denom = np.maximum(np.abs(r), floor)
        rel = np.abs(g - r) / denom
        bad = ~(rel <= rtol)
        rep[k] = dict(n=r.size, nbad=int(bad.sum()), max_rel=float(np.nanmax(rel)), bad=bad)
    return rep


def parity_summary(rep, shape2d, margins_ulps=None):
    """Columns failing tolerance, and how many of them sit near a threshold (trigger flips)."""
    cols = np.zeros(shape2d, bool)
    for v in rep.values():
        cols |= column_mask(v["bad"], shape2d)
    out = dict(bad_columns=int(cols.sum()), columns=int(np.prod(shape2d)))
    if margins_ulps is not None:
        near = cols & (margins_ulps <= 64)
        out["flip_columns"] = int(near.sum())
        out["unexplained_columns"] = int((cols & ~(margins_ulps <= 64)).sum())
        out["max_margin_ulps_of_bad"] = float(np.max(margins_ulps[cols])) if cols.any() else 0.0
    return out
