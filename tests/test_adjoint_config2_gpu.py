"""The adjoint workload at T42: 128 x 64 = 8,192 columns at 8 levels (land, orography, snow and
sea ice), the 12 differentiated tuning parameters (params.py:11-16, 51-54, 72-73) each scaled
by a seeded U(0.8, 1.2) factor, an N(0, 1) cotangent on every tendency output.

The GPU VJP (spd_vjp, float32) is compared column by column with the host builds of the same
reverse pass (tests/host/host_column.cpp) in float64 and float32, whose float64 VJP is the one
checked against central differences (tests/test_adjoint_cpu.py, tests/test_rollout_cpu.py).

Bars:
* state gradients, per field: |gpu - host| <= 1e-4 max|host| (normwise) against the float64 host
  VJP and against the float32 host VJP (the same float32 arithmetic, as jax.vjp of the float32
  reference would be).  A column where float32 takes another branch than float64 (a convection,
  condensation or cloud threshold) is a flip; flips are excluded from the float64 comparison and
  counted (at most 1 % of the columns).  The elementwise error above a floor of 1e-2 max|host|
  is reported beside it: like the forward's temperature tendency, these gradients are sums of
  cancelling terms, and the float32 host itself sits up to ~2e-4 elementwise from float64 there.
* parameter gradients: each of the 12 within 1e-4 relative of the float32 host sum over the
  columns, and of the float64 host sum with the flipped columns' contributions taken from the
  float32 host (they follow the float32 branch the GPU takes).
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from tests.test_adjoint_cpu import (VJP_HAND32, VJP_HAND64, HostColumn, _flags, build_host,
                                    column_of)
from oracle import speedy_oracle as O

pytestmark = pytest.mark.gpu

DIFF_GROUPS = {"psmin": "convection", "trcnv": "convection", "rhil": "convection",
               "rhbl": "convection", "entmax": "convection", "smf": "convection",
               "trlsc": "condensation", "rhlsc": "condensation", "drhlsc": "condensation",
               "rhblsc": "condensation", "albcl": "shortwave_radiation",
               "albcls": "shortwave_radiation"}
RTOL = 1e-4
ADJ_FLOOR = 1e-2
FLIP_FRAC = 1e-2


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    lib = build_host(tmp_path_factory.mktemp("hostcol2") / "libhostcol.so")
    d = C.POINTER(C.c_double)
    lib.hc_vjp_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.POINTER(HostColumn),
                                 C.c_int, d, d, C.c_double, C.c_double]
    lib.hc_vjp_batch.restype = C.c_int
    return lib


def perturbed_parameters(pkg, seed):
    """The 12 differentiated scalars, each times a seeded U(0.8, 1.2) factor."""
    rng = np.random.default_rng(seed)
    base = pkg.Parameters.default()
    out = {}
    for name, group in DIFF_GROUPS.items():
        v = float(np.float32(getattr(getattr(base, group), name) * rng.uniform(0.8, 1.2)))
        out[f"{group}.{name}"] = v
    return out


def host_vjp(host, vg, pr, cols, cts, mode):
    n = len(cols)
    arr = (HostColumn * n)(*cols)
    ct = np.ascontiguousarray(cts, np.float64)
    out = np.zeros((n, 63), np.float64)
    rc = host.hc_vjp_batch(mode, C.byref(vg), C.byref(pr), arr, n,
                           ct.ctypes.data_as(C.POINTER(C.c_double)),
                           out.ctypes.data_as(C.POINTER(C.c_double)), 1800.0, 1.0)
    assert rc == n, rc
    return out


def test_t42_adjoint_with_perturbed_parameters(pkg, host):
    import torch
    inst = pkg.synthetic.land_instance(42, 128, 64, 8, sst_noise=1.5)
    kx, ix, il = inst.kx, inst.ix, inst.il
    params = perturbed_parameters(pkg, seed=6)
    # the level set and per-latitude solar rows, from the float32 oracle with these parameters
    tend, data = O.compute_tendencies(*inst.oracle_args(O.default_parameters(**params)))
    S = int(sum(1 << int(l) for l in np.nonzero(O.cloud_top_level_set(
        data.shortwave_rad.icltop, kx))[0]))
    phys_params = pkg.Parameters.default().with_values(
        **{k.replace(".", "__"): v for k, v in params.items()})
    vg = pkg._lib.VGrid()
    vt = pkg.physics.initialize_vertical(kx)
    for name, a in zip(("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp"), vt[:6]):
        tgt = getattr(vg, name)
        for i, v in enumerate(a):
            tgt[i] = float(v)
    for k in range(kx):
        vg.wvi[k][0], vg.wvi[k][1] = float(vt[6][k, 0]), float(vt[6][k, 1])
    pr = phys_params.to_struct()

    rng = np.random.default_rng(7)
    shape = (kx, ix, il)
    cts = {k: rng.normal(size=shape).astype(np.float32) for k in ("u", "v", "t", "q")}
    state, forcing, geom, date = pkg.instance_to_device(inst, "cuda")
    phys = pkg.SpeedyPhysics(phys_params, diagnostics=False)
    t = lambda a: torch.as_tensor(a, dtype=torch.float32, device="cuda")
    cot = pkg.PhysicsTendency(t(cts["u"]), t(cts["v"]), t(cts["t"]), t(cts["q"]))
    gs, gp = pkg.adjoint.vjp(phys, state, forcing, geom, date, cot)
    torch.cuda.synchronize()
    c = lambda x: x.cpu().numpy().astype(np.float64)
    gpu = dict(t=c(gs.temperature), q=c(gs.specific_humidity), phi=c(gs.geopotential),
               psa=c(gs.normalized_surface_pressure)[None], u=c(gs.u_wind)[-1:],
               v=c(gs.v_wind)[-1:])
    p_gpu = c(gp)

    flags = _flags(inst)
    cols, ct_rows = [], []
    for i in range(ix):
        for j in range(il):
            cols.append(column_of(inst, data, S, i, j, flags))
            row = np.zeros(34)
            row[:kx] = cts["t"][:, i, j]
            row[16:16 + kx] = cts["q"][:, i, j]
            row[32], row[33] = cts["u"][-1, i, j], cts["v"][-1, i, j]
            ct_rows.append(row)
    h64 = host_vjp(host, vg, pr, cols, ct_rows, VJP_HAND64)
    h32 = host_vjp(host, vg, pr, cols, ct_rows, VJP_HAND32)

    def planes(h):
        r = lambda a, n: a.reshape(ix, il, n).transpose(2, 0, 1)
        return dict(t=r(h[:, 0:kx], kx), q=r(h[:, 16:16 + kx], kx), phi=r(h[:, 32:32 + kx], kx),
                    psa=r(h[:, 48:49], 1), u=r(h[:, 49:50], 1), v=r(h[:, 50:51], 1))

    H64, H32 = planes(h64), planes(h32)
    colmax = lambda e: e.reshape(-1, ix, il).max(axis=0)
    flips = np.zeros((ix, il), bool)
    report = {}
    for k in H64:
        s64 = max(np.max(np.abs(H64[k])), 1e-30)
        e32 = colmax(np.abs(H32[k] - H64[k])) / s64
        flips |= e32 > 1e-3  # float32 and float64 took different branches in this column
    keep = ~flips
    for k in H64:
        g, a, b = gpu[k], H32[k], H64[k]
        s32 = max(np.max(np.abs(a)), 1e-30)
        s64 = max(np.max(np.abs(b)), 1e-30)
        e_el = np.abs(g - a) / np.maximum(np.abs(a), ADJ_FLOOR * s32)
        e_el = colmax(e_el)
        e32 = colmax(np.abs(g - a)) / s32
        e64 = colmax(np.abs(g - b)) / s64
        e3264 = colmax(np.abs(a - b)) / s64
        report[k] = dict(norm_vs_f32=float(e32.max()), norm_vs_f64=float(e64[keep].max()),
                         f32_host_norm_vs_f64=float(e3264[keep].max()),
                         elem_vs_f32=float(e_el.max()))
    # parameter gradients: float32 host sum and the float64 sum with flipped columns taken
    # from the float32 host
    pc64, pc32 = h64[:, 51:63], h32[:, 51:63]
    fl = flips.reshape(-1)
    p32 = pc32.sum(axis=0)
    p64 = np.where(fl[:, None], pc32, pc64).sum(axis=0)
    p64_pure = pc64.sum(axis=0)
    rel32 = np.abs(p_gpu - p32) / np.maximum(np.abs(p32), 1e-30)
    rel64 = np.abs(p_gpu - p64) / np.maximum(np.abs(p64), 1e-30)
    cond = np.abs(pc64).sum(axis=0) / np.maximum(np.abs(p64_pure), 1e-30)
    names = list(DIFF_GROUPS)
    print("T42 perturbed", {k: {a: f"{b:.1e}" for a, b in v.items()} for k, v in report.items()},
          "flip columns", int(flips.sum()))
    print("params rel vs f32 host", dict(zip(names, (f"{x:.1e}" for x in rel32))))
    print("params rel vs f64 host", dict(zip(names, (f"{x:.1e}" for x in rel64))))
    print("params sum|c|/|sum|", dict(zip(names, (f"{x:.1e}" for x in cond))))
    assert flips.sum() <= FLIP_FRAC * ix * il
    for k, r in report.items():
        assert r["norm_vs_f32"] <= RTOL, (k, r)
        assert r["norm_vs_f64"] <= RTOL, (k, r)
    assert np.all(rel32 <= RTOL), dict(zip(names, rel32))
    assert np.all(rel64 <= RTOL), dict(zip(names, rel64))
