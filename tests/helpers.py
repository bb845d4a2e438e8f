"""Shared helpers of the parity tests: run an Instance through the CUDA path (via the C ABI)
and compare with the oracle under the stated tolerance."""
from __future__ import annotations

import numpy as np

# Parity bar, per field f:  |cuda - oracle32| <= RTOL * max|oracle32_f|  (normwise, i.e. a
# per-field absolute floor of RTOL * max|f|).  The float32 oracle itself sits at ~5e-6 of
# max|f| from the float64 oracle on these fields: the tendencies are sums of terms that cancel,
# so an elementwise 1e-5 bar would sit below float32's own rounding noise.  In addition the
# CUDA path's error against the float64 oracle must not exceed X64_FACTOR times the float32
# oracle's own error against float64, or within X64_FLOOR * max|f|.
#
# Diagnostic fields (cloud cover, surface radiation) carry more float32 noise than the
# tendencies: cloud cover takes sqrt of a precipitation rate that is ~0 in most columns, so the
# float32 oracle itself sits up to ~5e-5 of max|f| from float64 there.  Their bar is
# max(RTOL, NOISE_FACTOR * that float32-vs-float64 error), measured on the same inputs.  Their
# float64 check runs the float64 oracle on the CUDA path's own precipitation
# (conditional_diagnostics64), so that it tests the cloud and radiation arithmetic rather than
# sqrt's magnification of precipitation rounding.
RTOL = 1e-5
NOISE_FACTOR = 2.0
X64_FACTOR = 3.0
X64_FLOOR = 1e-5
STRICT_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "precnv", "precls")
DIAG_FIELDS = ("cloudc", "rsds", "rlds")
FLOAT_FIELDS = STRICT_FIELDS + DIAG_FIELDS


def to_device(pkg, inst, device="cuda"):
    return pkg.instance_to_device(inst, device)


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


def oracle_f64(inst):
    """The float64 oracle on the same (float32) input values: state, forcing and geometry
    fields are widened, vertical tables and parameters are rebuilt in float64."""
    from oracle import speedy_oracle as O
    a32 = inst.oracle_args(O.default_parameters())
    st, fo, ge, da, _ = O.cast_inputs(*a32, np.float64)
    for n, v in zip(("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp", "wvi"),
                    O.vertical_tables(inst.kx, np.float64)):
        setattr(ge, n, v)
    return st, fo, ge, da, O.default_parameters(np.float64)


def normwise(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def compare_fields(got, tend, data, ref64=None, rtol=RTOL):
    """Per-field report: normwise error, the tolerance applied and the elementwise failure
    mask.  ``ref64`` (the float64 oracle's (tend, data)) sets the diagnostic fields' noise-aware
    tolerance."""
    ref = oracle_fields(tend, data)
    r64 = oracle_fields(*ref64) if ref64 is not None else None
    rep = {}
    for k, r in ref.items():
        if k not in got:
            continue
        g = np.asarray(got[k], np.float64)
        r = np.asarray(r, np.float64)
        if k in ("icltop", "iptop"):
            bad = g != r
            rep[k] = dict(n=r.size, nbad=int(bad.sum()), norm=float(bad.mean()), tol=0.0, bad=bad)
            continue
        tol = rtol
        if k in DIAG_FIELDS and r64 is not None:
            tol = max(rtol, NOISE_FACTOR * normwise(r, r64[k]))
        scale = max(np.max(np.abs(r)), 1e-30)
        err = np.abs(g - r)
        bad = ~(err <= tol * scale)
        rep[k] = dict(n=r.size, nbad=int(bad.sum()), norm=float(np.nanmax(err) / scale),
                      tol=tol, bad=bad)
    return rep


def conditional_diagnostics64(inst, got, fuse_verify=False):
    """The float64 oracle with the CUDA path's precipitation substituted after the condensation
    term.  Cloud cover takes sqrt(precip) (shortwave_radiation.py:378), which magnifies the
    float32 rounding of a small precipitation rate without bound, and the surface radiation
    follows the cloud cover; evaluated on the precipitation the CUDA path produced (itself held
    to the 1e-5 bar), these diagnostics test the cloud and radiation arithmetic alone."""
    from oracle import speedy_oracle as O
    st, fo, ge, da, p = oracle_f64(inst)
    if fuse_verify:
        st = O.verify_state(st)
    kx, ix, il = st.temperature.shape
    data = O.zeros_data((ix, il), kx, da, np.float64)
    f2 = O.forcing_day_slice(fo, da)
    for term in O.TERMS:
        _, data = term(st, data, p, f2, ge)
        if term is O.get_large_scale_condensation_tendencies:
            data.convection.precnv = np.asarray(got["precnv"], np.float64)
            data.condensation.precls = np.asarray(got["precls"], np.float64)
    return data


def x64_errors(got, tend, data, ref64, exclude_cols=None, cond64=None):
    """Normwise errors of the CUDA path and of the float32 oracle against the float64 oracle,
    over the columns not in ``exclude_cols`` (trigger flips).  With ``cond64`` (the data of
    ``conditional_diagnostics64``) the CUDA path's diagnostic fields are measured against it."""
    ref = oracle_fields(tend, data)
    r64 = oracle_fields(*ref64)
    c64 = oracle_fields(ref64[0], cond64) if cond64 is not None else r64
    out = {}
    for k in FLOAT_FIELDS:
        if k not in got:
            continue
        g, r, x = (np.asarray(a, np.float64) for a in (got[k], ref[k], r64[k]))
        xc = np.asarray(c64[k] if k in DIAG_FIELDS else r64[k], np.float64)
        if exclude_cols is not None and exclude_cols.any():
            keep = ~exclude_cols
            g, r, x, xc = g[..., keep], r[..., keep], x[..., keep], xc[..., keep]
        s64 = max(np.max(np.abs(x)), 1e-30)
        out[k] = (float(np.max(np.abs(g - xc)) / s64), float(np.max(np.abs(r - x)) / s64))
    return out


def x64_violations(errs):
    return {k: v for k, v in errs.items() if v[0] > max(X64_FLOOR, X64_FACTOR * v[1])}


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
    out["_cols"] = cols
    return out


def parity_check(pkg, inst, params=None, max_flip_frac=2e-3, device="cuda", **kw):
    """Run ``inst`` through the CUDA path and hold it to the parity bar against the float32
    and float64 oracles; returns the per-field report and the column summary."""
    from oracle import speedy_oracle as O
    got = run_gpu_instance(pkg, inst, device=device, params=params, **kw)
    args = list(inst.oracle_args(O.default_parameters()))
    rec = O.Margins((inst.ix, inst.il))
    step = O.physics_step if kw.get("fuse_verify") else O.compute_tendencies
    oro = bool(kw.get("orographic_correction"))
    tend, data = step(*args, rec=rec, orographic=oro)
    ref64 = step(*oracle_f64(inst), orographic=oro)
    rep = compare_fields(got, tend, data, ref64)
    summ = parity_summary(rep, (inst.ix, inst.il), rec.ulps)
    cols = summ.pop("_cols")
    cond = conditional_diagnostics64(inst, got, fuse_verify=bool(kw.get("fuse_verify")))
    x64 = x64_errors(got, tend, data, ref64, exclude_cols=cols, cond64=cond)
    print(inst.name, {k: (v["nbad"], f"{v['norm']:.1e}") for k, v in rep.items()}, summ,
          {k: (f"{a:.1e}", f"{b:.1e}") for k, (a, b) in x64.items()})
    assert summ["unexplained_columns"] == 0, (summ, {k: v["nbad"] for k, v in rep.items()})
    assert summ["flip_columns"] <= max(2, max_flip_frac * summ["columns"]), summ
    assert not x64_violations(x64), x64_violations(x64)
    return rep, summ


def fake_fields(L, base=1 << 36, spacing=1 << 28):
    """Inputs and Outputs structs of distinct, non-overlapping, aligned fake device addresses
    (one `spacing`-sized slot per field), for argument checks that return before any device
    work and never dereference them."""
    n_in = len(L.INPUT_FIELDS)
    inp = L.Inputs(**{k: base + i * spacing for i, k in enumerate(L.INPUT_FIELDS)})
    out = L.Outputs(**{k: base + (n_in + i) * spacing for i, k in enumerate(L.OUTPUT_FIELDS)})
    return inp, out
