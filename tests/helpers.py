"""Shared helpers of the parity tests: run an Instance through the CUDA path (via the C ABI)
and compare with the oracle under the stated tolerance."""
from __future__ import annotations

import numpy as np

# Parity bar, per output field f, element by element:
#
#     |cuda - oracle32| <= RTOL * max(|oracle32|, ELEM_FLOOR[f] * max|oracle32_f|)
#
# i.e. relative error RTOL = 1e-5 above a per-field absolute floor.  Integer levels (iptop,
# icltop) must match exactly.  Columns outside the bar must be trigger flips: a threshold test
# of that column sits within FLIP_ULPS float32 ulps of its threshold in the oracle (counted by
# ulp bucket -- within 1, within 4, within 64 -- and bounded).  The floors follow the float32
# conditioning of each field.  The winds and the large-scale precipitation take 1e-3.  The
# temperature and humidity tendencies and the convective precipitation are sums of radiative,
# convective and diffusive terms that cancel: two float32 evaluations of the reference
# arithmetic that differ only in the last bits of their exponentials already need floors of up
# to 0.56 (temperature), 0.41 (humidity) and 0.36 (convective precipitation) of the field
# maximum to agree within 1e-5 (tests/test_float32_sensitivity.py, and the same measurement on
# the T425 instance), and the CUDA path needs at most 0.80, 0.48 and 0.41 over every GPU parity
# case (T425 included); their floors are 1.0, 0.5 and 0.5 -- for the temperature tendency the
# elementwise bar is the normwise one.  Normwise error <= RTOL * max|f| is asserted for every
# field as well, and the CUDA path's error against the float64 oracle must stay within
# max(X64_FLOOR, X64_FACTOR x the float32 oracle's own).
#
# Diagnostic fields (cloud cover, surface radiation) carry more float32 noise than the
# tendencies: cloud cover takes sqrt of a precipitation rate that is ~0 in most columns, so the
# float32 oracle itself sits up to ~5e-5 of max|f| from float64 there.  Their bar is normwise,
# max(RTOL, NOISE_FACTOR * that float32-vs-float64 error), measured on the same inputs.  Their
# float64 check runs the float64 oracle on the CUDA path's own precipitation
# (conditional_diagnostics64), so that it tests the cloud and radiation arithmetic rather than
# sqrt's magnification of precipitation rounding.  Their elementwise figures are reported.
RTOL = 1e-5
ELEM_FLOOR = {"u_wind": 1e-3, "v_wind": 1e-3, "precnv": 0.5, "precls": 1e-3,
              "temperature": 1.0, "specific_humidity": 0.5}
REPORT_FLOOR = 1e-3  # the floor at which elementwise counts are also reported for every field
FLIP_ULPS = 64
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


def oracle_args(inst, params=None):
    """The oracle's (state, forcing, geometry, date, params) for ``inst``; ``params`` is a dict
    of parameter overrides keyed ``"group.name"`` (the oracle's naming)."""
    from oracle import speedy_oracle as O
    return inst.oracle_args(O.default_parameters(**(params or {})))


def oracle_f64(inst, params=None):
    """The float64 oracle on the same (float32) input values: state, forcing and geometry
    fields are widened, vertical tables and parameters are rebuilt in float64."""
    from oracle import speedy_oracle as O
    a32 = oracle_args(inst, params)
    st, fo, ge, da, _ = O.cast_inputs(*a32, np.float64)
    for n, v in zip(("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp", "wvi"),
                    O.vertical_tables(inst.kx, np.float64)):
        setattr(ge, n, v)
    return st, fo, ge, da, O.default_parameters(np.float64, **(params or {}))


def normwise(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30))


def elementwise(g, r, floor):
    """Elementwise relative error |g - r| / max(|r|, floor * max|r|)."""
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    scale = max(np.max(np.abs(r)), 1e-30)
    return np.abs(g - r) / np.maximum(np.abs(r), floor * scale)


def required_floor(g, r, keep=None, rtol=RTOL):
    """The smallest floor (fraction of max|r|) at which every element (of the columns in
    ``keep``) meets relative error rtol: max over elements with |g-r| > rtol |r| of
    |g-r| / (rtol max|r|)."""
    g = np.asarray(g, np.float64)
    r = np.asarray(r, np.float64)
    if keep is not None:
        g, r = g[..., keep], r[..., keep]
    if g.size == 0:
        return 0.0
    d = np.abs(g - r)
    scale = max(np.max(np.abs(r)), 1e-30)
    over = d > rtol * np.abs(r)
    return float(np.max(d[over]) / (rtol * scale)) if over.any() else 0.0


def compare_fields(got, tend, data, ref64=None, rtol=RTOL):
    """Per-field report: normwise error, the elementwise error above the field's floor, the
    tolerance applied and the elementwise failure mask.  ``ref64`` (the float64 oracle's
    (tend, data)) sets the diagnostic fields' noise-aware normwise tolerance."""
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
        scale = max(np.max(np.abs(r)), 1e-30)
        err = np.abs(g - r)
        e_rep = elementwise(g, r, REPORT_FLOOR)
        item = dict(n=r.size, norm=float(np.nanmax(err) / scale),
                    elem_n_over_at_1e3=int((~(e_rep <= rtol)).sum()),
                    elem_max_at_1e3=float(np.nanmax(e_rep)))
        if k in DIAG_FIELDS:
            tol = rtol
            if r64 is not None:
                tol = max(rtol, NOISE_FACTOR * normwise(r, r64[k]))
            bad = ~(err <= tol * scale)
            item.update(tol=tol, bad=bad, kind="normwise")
        else:
            floor = ELEM_FLOOR[k]
            e = elementwise(g, r, floor)
            bad = ~(e <= rtol)
            item.update(tol=rtol, floor=floor, elem_max=float(np.nanmax(e)), bad=bad,
                        bad_norm=~(err <= rtol * scale), kind="elementwise")
        item["nbad"] = int(bad.sum())
        rep[k] = item
    return rep


def conditional_diagnostics64(inst, got, fuse_verify=False, params=None):
    """The float64 oracle with the CUDA path's precipitation substituted after the condensation
    term.  Cloud cover takes sqrt(precip) (shortwave_radiation.py:378), which magnifies the
    float32 rounding of a small precipitation rate without bound, and the surface radiation
    follows the cloud cover; evaluated on the precipitation the CUDA path produced (itself held
    to the 1e-5 bar), these diagnostics test the cloud and radiation arithmetic alone."""
    from oracle import speedy_oracle as O
    st, fo, ge, da, p = oracle_f64(inst, params)
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
        if g.size == 0:  # every column is a counted flip
            continue
        s64 = max(np.max(np.abs(x)), 1e-30)
        out[k] = (float(np.max(np.abs(g - xc)) / s64), float(np.max(np.abs(r - x)) / s64))
    return out


def x64_violations(errs):
    return {k: v for k, v in errs.items() if v[0] > max(X64_FLOOR, X64_FACTOR * v[1])}


def parity_summary(rep, shape2d, margins_ulps=None):
    """Columns failing the bar, and how many of them sit near a threshold (trigger flips),
    counted by the oracle's smallest threshold margin: within 1 ulp, within 4, within
    FLIP_ULPS; the rest are unexplained."""
    cols = np.zeros(shape2d, bool)
    for v in rep.values():
        cols |= column_mask(v["bad"], shape2d)
    out = dict(bad_columns=int(cols.sum()), columns=int(np.prod(shape2d)))
    if margins_ulps is not None:
        m = np.asarray(margins_ulps)
        near = cols & (m <= FLIP_ULPS)
        out["flip_columns"] = int(near.sum())
        out["flip_columns_le_1ulp"] = int((cols & (m <= 1)).sum())
        out["flip_columns_1_to_4ulp"] = int((cols & (m > 1) & (m <= 4)).sum())
        out["flip_columns_4_to_64ulp"] = int((cols & (m > 4) & (m <= FLIP_ULPS)).sum())
        out["unexplained_columns"] = int((cols & ~(m <= FLIP_ULPS)).sum())
        out["max_margin_ulps_of_bad"] = float(np.max(m[cols])) if cols.any() else 0.0
    out["_cols"] = cols
    return out


def oracle_step(kw):
    from oracle import speedy_oracle as O
    return O.physics_step if kw.get("fuse_verify") else O.compute_tendencies


def oracle_kwargs(kw):
    """The oracle-side keyword arguments of a SpeedyPhysics configuration."""
    out = dict(orographic=bool(kw.get("orographic_correction")))
    if kw.get("fuse_verify"):
        if kw.get("time_step") is not None:
            out["time_step"] = kw["time_step"]
    return out


def apply_q_scale(tend, scale):
    """The humidity tendency unit scale the kernel fuses last (physics_interface.py:286)."""
    if scale is not None and scale != 1.0:
        dt = tend.specific_humidity.dtype.type
        tend.specific_humidity = (tend.specific_humidity * dt(scale)).astype(
            tend.specific_humidity.dtype)
    return tend


def check_against_oracle(inst, got, params=None, max_flip_frac=2e-3, label=None, **kw):
    """Holds the CUDA results ``got`` of ``inst`` to the parity bar against the float32 and
    float64 oracles; returns the per-field report and the column summary."""
    from oracle import speedy_oracle as O
    args = list(oracle_args(inst, params))
    rec = O.Margins((inst.ix, inst.il))
    step = oracle_step(kw)
    okw = oracle_kwargs(kw)
    tend, data = step(*args, rec=rec, **okw)
    tend64, data64 = step(*oracle_f64(inst, params), **okw)
    qs = kw.get("q_tend_scale")
    tend, tend64 = apply_q_scale(tend, qs), apply_q_scale(tend64, qs)
    rep = compare_fields(got, tend, data, (tend64, data64))
    summ = parity_summary(rep, (inst.ix, inst.il), rec.ulps)
    cols = summ.pop("_cols")
    cond = conditional_diagnostics64(inst, got, fuse_verify=bool(kw.get("fuse_verify")),
                                     params=params)
    x64 = x64_errors(got, tend, data, (tend64, data64), exclude_cols=cols, cond64=cond)
    keep = ~cols
    norm_bad = {k: int(column_mask(v["bad_norm"], cols.shape)[keep].sum())
                for k, v in rep.items() if "bad_norm" in v}
    floors = {k: round(required_floor(got[k], oracle_fields(tend, data)[k], keep), 4)
              for k in STRICT_FIELDS if k in got}
    print(label or inst.name,
          {k: (v["nbad"], f"{v['norm']:.1e}", f"e{v.get('elem_max', 0):.1e}",
               v["elem_n_over_at_1e3"]) for k, v in rep.items() if k in FLOAT_FIELDS},
          {k: v for k, v in summ.items()},
          "required floors", floors,
          {k: (f"{a:.1e}", f"{b:.1e}") for k, (a, b) in x64.items()})
    assert summ["unexplained_columns"] == 0, (summ, {k: v["nbad"] for k, v in rep.items()})
    assert summ["flip_columns"] <= max(2, max_flip_frac * summ["columns"]), summ
    assert not any(norm_bad.values()), norm_bad
    assert not x64_violations(x64), x64_violations(x64)
    summ["required_floors"] = floors
    return rep, summ


def parity_check(pkg, inst, params=None, max_flip_frac=2e-3, device="cuda", **kw):
    """Run ``inst`` through the CUDA path and hold it to the parity bar against the float32
    and float64 oracles; returns the per-field report and the column summary."""
    phys_params = None
    if params:
        phys_params = pkg.Parameters.default().with_values(
            **{k.replace(".", "__"): v for k, v in params.items()})
    got = run_gpu_instance(pkg, inst, device=device, params=phys_params, **kw)
    return check_against_oracle(inst, got, params=params, max_flip_frac=max_flip_frac, **kw)


def fake_fields(L, base=1 << 36, spacing=1 << 28):
    """Inputs and Outputs structs of distinct, non-overlapping, aligned fake device addresses
    (one `spacing`-sized slot per field), for argument checks that return before any device
    work and never dereference them."""
    n_in = len(L.INPUT_FIELDS)
    inp = L.Inputs(**{k: base + i * spacing for i, k in enumerate(L.INPUT_FIELDS)})
    out = L.Outputs(**{k: base + (n_in + i) * spacing for i, k in enumerate(L.OUTPUT_FIELDS)})
    return inp, out
