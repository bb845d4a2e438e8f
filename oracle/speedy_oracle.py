"""Oracle: a NumPy restatement of JAX-GCM's SPEEDY column physics.

TEST INFRASTRUCTURE ONLY.  This module is the parity checker for the CUDA path.  Only
``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product path (``jax-gcm_b200``) never calls it and
fails loudly when its CUDA library is missing.

Every function restates one reference function and cites it as ``file:line`` relative to the
JAX-GCM project root (``jcm/...``).  Arrays keep the reference layout ``[kx, ix, il]`` (2-D
fields ``[ix, il]``, per-latitude tables ``[il]``) so the reference's own unit tests port
one-to-one.  The arithmetic follows the reference expression by expression, including its
quirks (the shortwave cloud-top level set, the LSC ``iptop`` rule, dropped out-of-range
scatters, the SW->LW ``flux`` hand-off).  ``dtype`` selects float32 (the parity target) or
float64 (the x64 error report).  NumPy 2 follows NEP 50, so Python float constants are weak
and combine with float32 arrays in float32, exactly like JAX's weak typing.

Pinning: ``tests/test_oracle_goldens.py`` checks these functions against every golden vector
and known-answer test the reference ships for this path (the Fortran-derived ``.npy`` arrays
and the literal arrays in ``jcm/physics/speedy/*_test.py``), extracted by
``tests/golden/make_golden.py``.
"""
from __future__ import annotations

import copy as _copy
from types import SimpleNamespace

import numpy as np

# ---------------------------------------------------------------------------------------------
# Constants: jcm/constants.py:3-5, jcm/physics/speedy/physical_constants.py:9-51,
# jcm/physics/speedy/physics_data.py:6, jcm/physics/speedy/forcing.py:8, jcm/date.py:6
# ---------------------------------------------------------------------------------------------
P0 = 1e5
GRAV = 9.81
CP = 1004.0
AKAP = 2.0 / 7.0
RGAS = AKAP * CP
ALHC = 2501.0
ALHS = 2801.0
SBC = 5.67e-8
SOLC = 342.0
EPSSW = 0.020
SD2SC = 60.0
EPSILON = 1e-9
NSTRAD = 3
ABLCO2_REF = 6.0
DEL_CO2 = 0.005
DAYS_YEAR = 365.2425

# physical_constants.py:47-51; 16 uniform levels are the kx-generic extension used by the
# 16-level workloads (the physics arithmetic itself is kx-generic).
SIGMA_LAYER_BOUNDARIES = {
    7: [0.0, 0.14, 0.26, 0.42, 0.6, 0.77, 0.9, 1.0],
    8: [0.0, 0.05, 0.14, 0.26, 0.42, 0.6, 0.77, 0.9, 1.0],
    16: [k / 16.0 for k in range(17)],
}


# ---------------------------------------------------------------------------------------------
# Exponential hook.  Every exp of the physics goes through exp_.  By default it is np.exp.
# Inside ``perturbed_exp`` each float32 result is multiplied by (1 + r 2^-23), with r drawn
# uniformly from (-ulps, ulps) per element.  Library exps differ from one another in their last
# bits, and this is Monte Carlo arithmetic (D. Stott Parker, 1997) applied to the one operation
# whose rounding differs between float32 implementations.  Re-running the float32 oracle under it
# measures, per output element, how far last-bit differences in the transcendentals move that
# element.  The parity tests use this to tell float32 noise from a wrong result.
# ---------------------------------------------------------------------------------------------
_EXP_NOISE = None  # (numpy Generator, ulps) while perturbed_exp is active


def exp_(x):
    y = np.exp(x)
    if _EXP_NOISE is None or np.asarray(y).dtype != np.float32:
        return y
    rng, ulps = _EXP_NOISE
    ya = np.asarray(y)
    r = rng.uniform(-ulps, ulps, ya.shape)
    z = (ya.astype(np.float64) * (1.0 + r * 2.0 ** -23)).astype(np.float32)
    return z if isinstance(y, np.ndarray) else np.float32(z)


class perturbed_exp:
    """Context manager: float32 exp results carry a seeded relative noise of up to ``ulps``."""

    def __init__(self, seed, ulps=2.0):
        self.noise = (np.random.default_rng(seed), float(ulps))

    def __enter__(self):
        global _EXP_NOISE
        self.prev, _EXP_NOISE = _EXP_NOISE, self.noise
        return self

    def __exit__(self, *exc):
        global _EXP_NOISE
        _EXP_NOISE = self.prev
        return False


def ns(**kw):
    return SimpleNamespace(**kw)


# ---------------------------------------------------------------------------------------------
# Parameters: jcm/physics/speedy/params.py:9-254 (defaults)
# ---------------------------------------------------------------------------------------------
PARAM_DEFAULTS = {
    "convection": dict(psmin=0.8, trcnv=6.0, rhil=0.7, rhbl=0.9, entmax=0.5, smf=0.8),
    "condensation": dict(trlsc=4.0, rhlsc=0.9, drhlsc=0.1, rhblsc=0.95),
    "shortwave_radiation": dict(
        albcl=0.43, albcls=0.50, absdry=0.033, absaer=0.033, abswv1=0.022, abswv2=15.000,
        abscl1=0.015, abscl2=0.15, ablwin=0.3, ablwv1=0.7, ablwv2=50.0, ablcl1=12.0,
        ablcl2=0.6, rhcl1=0.30, rhcl2=1.00, qacl=0.20, wpcl=0.2, pmaxcl=10.0, clsmax=0.60,
        clsminl=0.15, gse_s0=0.25, gse_s1=0.40),
    "mod_radcon": dict(albsea=0.07, albice=0.60, albsn=0.60, epslw=0.05, emisfc=0.98),
    "surface_flux": dict(
        fwind0=0.95, ftemp0=1.0, fhum0=0.0, cdl=2.4e-3, cds=1.0e-3, chl=1.2e-3, chs=0.9e-3,
        vgust=5.0, ctday=1.0e-2, dtheta=3.0, fstab=0.67, clambda=7.0, clambsn=7.0,
        hdrag=2000.0),
    "vertical_diffusion": dict(trshc=6.0, trvdi=24.0, trvds=6.0, redshc=0.5, rhgrad=0.5,
                               segrad=0.1),
}
PARAM_FLAGS = {"surface_flux": dict(lscasym=True, lskineb=True),
               "forcing": dict(increase_co2=False, co2_year_ref=1950)}

# The 12 scalars the adjoint differentiates (params.py:11-16, :51-54, :72-73).
DIFF_PARAMS = [("convection", "psmin"), ("convection", "trcnv"), ("convection", "rhil"),
               ("convection", "rhbl"), ("convection", "entmax"), ("convection", "smf"),
               ("condensation", "trlsc"), ("condensation", "rhlsc"),
               ("condensation", "drhlsc"), ("condensation", "rhblsc"),
               ("shortwave_radiation", "albcl"), ("shortwave_radiation", "albcls")]


def default_parameters(dtype=np.float32, **overrides):
    """Parameters.default() (params.py:244-254) with float leaves cast to ``dtype``."""
    groups = {}
    for g, d in PARAM_DEFAULTS.items():
        groups[g] = {k: dtype(v) for k, v in d.items()}
    for g, d in PARAM_FLAGS.items():
        groups.setdefault(g, {}).update(d)
    for key, val in overrides.items():
        g, k = key.split(".")
        groups[g][k] = val if isinstance(val, (bool, int, np.bool_)) and not isinstance(
            val, float) and k in ("lscasym", "lskineb", "increase_co2", "co2_year_ref") \
            else dtype(val)
    return ns(**{g: ns(**d) for g, d in groups.items()})


# ---------------------------------------------------------------------------------------------
# Geometry: jcm/geometry.py:62-85 (vertical), :130-132 (latitudes),
# jcm/physics/speedy/test_utils.py:4-16 (SPEEDY latitudes used by the reference unit tests)
# ---------------------------------------------------------------------------------------------
def vertical_tables(kx, dtype=np.float32):
    """_initialize_vertical (geometry.py:62-85), evaluated in ``dtype``."""
    hsg = np.asarray(SIGMA_LAYER_BOUNDARIES[kx], dtype=dtype)
    fsg = (hsg[1:] + hsg[:-1]) / 2.0
    dhs = np.diff(hsg)
    sigl = np.log(fsg)
    grdsig = GRAV / (dhs * P0)
    grdscp = grdsig / CP
    wvi = np.zeros((kx, 2), dtype=dtype)
    wvi[:-1, 0] = 1.0 / np.diff(sigl)
    wvi[:-1, 1] = (np.log(hsg[1:-1]) - sigl[:-1]) * wvi[:-1, 0]
    wvi[-1, 1] = (np.log(dtype(0.99)) - sigl[-1]) * wvi[-2, 0]
    return hsg, fsg, dhs, sigl, grdsig, grdscp, wvi


def gaussian_latitudes(il):
    """Gauss-Legendre latitudes south->north in radians (float64)."""
    x, _ = np.polynomial.legendre.leggauss(il)
    return np.arcsin(x)


def speedy_latitudes(il):
    """convert_to_speedy_latitudes (physics/speedy/test_utils.py:4-16), float64 then cast."""
    iy = (il + 1) // 2
    j = np.arange(1, iy + 1, dtype=np.float32)
    sia_half = np.cos(np.float32(np.pi) * (j - np.float32(0.25)) / np.float32(il + 0.5))
    radang = np.concatenate((-np.arcsin(sia_half), np.arcsin(sia_half)[::-1]))
    sia = np.concatenate((-sia_half, sia_half[::-1]))
    coa = np.cos(radang)
    return radang, sia, coa


def make_geometry(ix, il, kx, dtype=np.float32, lat="gaussian", orog=None, fmask=None,
                  phis0=None):
    """A Geometry (geometry.py:87-106) built without dinosaur.

    ``phis0`` defaults to ``grav*orog`` (the single-column rule, geometry.py:226-227); for the
    flat or constant orography of the reference tests the spectral truncation of
    geometry.py:128 leaves it unchanged.
    """
    hsg, fsg, dhs, sigl, grdsig, grdscp, wvi = vertical_tables(kx, dtype)
    if isinstance(lat, str) and lat == "gaussian":
        radang = gaussian_latitudes(il)
        sia, coa = np.sin(radang).astype(dtype), np.cos(radang).astype(dtype)
    elif isinstance(lat, str) and lat == "speedy":
        radang, sia, coa = speedy_latitudes(il)
        sia, coa = sia.astype(dtype), coa.astype(dtype)
    else:
        radang = np.asarray(lat, dtype=np.float64)
        sia, coa = np.sin(radang).astype(dtype), np.cos(radang).astype(dtype)
    orog = np.zeros((ix, il), dtype) if orog is None else np.broadcast_to(
        np.asarray(orog, dtype), (ix, il)).copy()
    fmask = np.zeros((ix, il), dtype) if fmask is None else np.broadcast_to(
        np.asarray(fmask, dtype), (ix, il)).copy()
    if phis0 is None:
        phis0 = (GRAV * orog).astype(dtype)
    return ns(nodal_shape=(kx, ix, il), orog=orog, phis0=np.asarray(phis0, dtype), fmask=fmask,
              radang=np.asarray(radang, dtype), sia=sia, coa=coa, hsg=hsg, fsg=fsg, dhs=dhs,
              sigl=sigl, grdsig=grdsig, grdscp=grdscp, wvi=wvi)


# ---------------------------------------------------------------------------------------------
# State / tendency / forcing / date / data containers
# ---------------------------------------------------------------------------------------------
def make_state(shape, dtype=np.float32, **fields):
    """PhysicsState.zeros (physics_interface.py:31-40)."""
    kx, ix, il = shape
    z3 = lambda: np.zeros(shape, dtype)
    st = ns(u_wind=z3(), v_wind=z3(), temperature=z3(), specific_humidity=z3(),
            geopotential=z3(), normalized_surface_pressure=np.zeros((ix, il), dtype))
    for k, v in fields.items():
        setattr(st, k, np.broadcast_to(np.asarray(v, dtype), getattr(st, k).shape).copy())
    return st


def zero_tendency(shape, dtype):
    z = lambda: np.zeros(shape, dtype)
    return ns(u_wind=z(), v_wind=z(), temperature=z(), specific_humidity=z())


def make_forcing(xy, dtype=np.float32, fill=0.0, lfluxland=None, **fields):
    """ForcingData.zeros / .ones (forcing.py:19-45)."""
    mk = lambda: np.full(xy, fill, dtype)
    f = ns(alb0=mk(), sice_am=mk(), snowc_am=mk(), soilw_am=mk(), stl_am=mk(),
           sea_surface_temperature=mk(),
           lfluxland=bool(fill) if lfluxland is None else bool(lfluxland))
    for k, v in fields.items():
        setattr(f, k, np.broadcast_to(np.asarray(v, dtype), xy).copy())
    return f


def make_date(tyear=0.0, model_year=1950, model_step=0, dt_seconds=1800.0, dtype=np.float32):
    """DateData.zeros (date.py:16-23)."""
    return ns(tyear=dtype(tyear), model_year=np.int32(model_year),
              model_step=np.int32(model_step), dt_seconds=dtype(dt_seconds))


def model_day(date):
    """DateData.model_day (date.py:40-41): round-half-even like jnp.round."""
    return int(np.round(np.float32(date.tyear) * np.float32(DAYS_YEAR)))


def zeros_data(xy, kx, date, dtype=np.float32, fill=0.0):
    """PhysicsData.zeros (physics_data.py:449-518) restated field by field."""
    f2 = lambda: np.full(xy, fill, dtype)
    f3 = lambda: np.full((kx,) + xy, fill, dtype)
    i2 = lambda: np.full(xy, int(fill), np.int64)
    return ns(
        shortwave_rad=ns(qcloud=f2(), fsol=f2(), rsds=f2(), rsns=f2(), ozone=f2(), ozupp=f2(),
                         zenit=f2(), stratz=f2(), gse=f2(), icltop=i2(), cloudc=f2(),
                         cloudstr=f2(), ftop=f2(), dfabs=f3(), compute_shortwave=bool(fill)),
        longwave_rad=ns(dfabs=f3(), ftop=f2()),
        mod_radcon=ns(ablco2=np.dtype(dtype).type(ABLCO2_REF), alb_l=f2(), alb_s=f2(), albsfc=f2(),
                      snowc=f2(), tau2=np.full((kx,) + xy + (4,), fill, dtype),
                      st4a=np.full((kx,) + xy + (2,), fill, dtype),
                      stratc=np.full(xy + (2,), fill, dtype),
                      flux=np.full(xy + (4,), fill, dtype)),
        condensation=ns(precls=f2(), dtlsc=f3(), dqlsc=f3()),
        convection=ns(se=f3(), iptop=i2(), cbmf=f2(), precnv=f2()),
        humidity=ns(rh=f3(), qsat=f3()),
        surface_flux=ns(ustr=np.full(xy + (3,), fill, dtype), vstr=np.full(xy + (3,), fill, dtype),
                        shf=np.full(xy + (3,), fill, dtype), evap=np.full(xy + (3,), fill, dtype),
                        rlus=np.full(xy + (3,), fill, dtype), rlds=f2(), rlns=f2(),
                        hfluxn=np.full(xy + (2,), fill, dtype), tsfc=f2(), tskin=f2(), u0=f2(),
                        v0=f2(), t0=f2()),
        date=date,
    )


def dcopy(x):
    return _copy.deepcopy(x)


class Margins:
    """Records, per column, the smallest distance (in float32 ulps) of any threshold test.

    A test is recorded between the two quantities it compares, on their own scale (a difference
    tested against zero is recorded between the terms it subtracts), so that the distance in
    ulps says how much rounding it takes to decide the test the other way.

    Columns whose CUDA result differs from the oracle beyond tolerance must have a trigger
    within a few ulps of its threshold (a "trigger flip"); the parity tests count them.
    """

    def __init__(self, xy):
        self.ulps = np.full(xy, np.inf)

    def cmp(self, a, b):
        a = np.asarray(a, np.float64)
        b = np.asarray(b, np.float64)
        scale = np.maximum(np.abs(a), np.abs(b))
        with np.errstate(all="ignore"):
            u = np.abs(a - b) / (scale * 2.0 ** -23)
        u = np.where(scale == 0.0, np.inf, u)  # 0 against 0: both sides exact, no threshold
        while u.ndim > len(self.ulps.shape):
            u = u.min(axis=0)
        u = np.broadcast_to(u, self.ulps.shape)
        self.ulps = np.minimum(self.ulps, np.where(np.isnan(u), np.inf, u))


def _rec(rec, a, b):
    if rec is not None:
        rec.cmp(a, b)


# ---------------------------------------------------------------------------------------------
# humidity.py
# ---------------------------------------------------------------------------------------------
def get_qsat(ta, ps, sig, rec=None):
    """get_qsat (humidity.py:73-104); ``sig > 0`` on every path the physics takes."""
    e0 = 6.108e-3
    c1 = 17.269
    c2 = 21.875
    t0 = 273.16
    t1 = 35.86
    t2 = 7.66
    with np.errstate(all="ignore"):
        _rec(rec, ta, t0)
        qsat = np.where(ta >= t0, e0 * exp_(c1 * (ta - t0) / (ta - t1)),
                        e0 * exp_(c2 * (ta - t0) / (ta - t2)))
        qsat = 622.0 * qsat / (sig * ps - 0.378 * qsat)
    return qsat


def rel_hum_to_spec_hum(ta, ps, sig, rh):
    """rel_hum_to_spec_hum (humidity.py:53-71)."""
    qsat = get_qsat(ta, ps, sig)
    return rh * qsat, qsat


def spec_hum_to_rel_hum(state, data, params, forcing, geometry, rec=None):
    """spec_hum_to_rel_hum (humidity.py:16-51)."""
    psa = state.normalized_surface_pressure
    qsat = get_qsat(state.temperature, psa[None], geometry.fsg[:, None, None], rec)
    with np.errstate(all="ignore"):
        rh = state.specific_humidity / qsat
    data = dcopy(data)
    data.humidity.rh = rh
    data.humidity.qsat = qsat
    return None, data


# ---------------------------------------------------------------------------------------------
# convection.py
# ---------------------------------------------------------------------------------------------
def diagnose_convection(psa, se, qa, qsat, params, forcing, geometry, rec=None):
    """diagnose_convection (convection.py:15-97)."""
    kx, ix, il = se.shape
    pc = params.convection
    iptop = np.full((ix, il), kx + 1, dtype=np.int64)
    qdif = np.zeros((ix, il), dtype=se.dtype)
    mss = se + ALHC * qsat
    rlhc = 1.0 / ALHC
    _rec(rec, psa, pc.psmin)
    mask_psa = psa > pc.psmin
    mse0 = se[kx - 1] + ALHC * qa[kx - 1]
    mse1 = se[kx - 2] + ALHC * qa[kx - 2]
    mse1 = np.minimum(mse0, mse1)
    mss0 = np.maximum(mse0, mss[kx - 1])
    mss2 = np.zeros_like(mss)
    mss2[:-1] = mss[:-1] + geometry.wvi[:-1, 1, None, None] * np.diff(mss, axis=0)
    levels = np.arange(2, kx - 3)

    def cloud_top(inst):
        return np.where(np.any(inst, axis=0), (levels + 1)[np.argmax(inst, axis=0)], kx)

    _rec(rec, mss0[None], mss2[2:kx - 3])
    ktop1 = cloud_top(mss0 > mss2[2:kx - 3])
    _rec(rec, mse1[None], mss2[2:kx - 3])
    ktop2 = cloud_top(mse1 > mss2[2:kx - 3])
    msthr = np.take_along_axis(mss2, (ktop2 - 1)[None], axis=0)[0]
    qthr0 = pc.rhbl * qsat[kx - 1]
    qthr1 = pc.rhbl * qsat[kx - 2]
    _rec(rec, qa[kx - 1], qthr0)
    _rec(rec, qa[kx - 2], qthr1)
    lqthr = (qa[kx - 1] > qthr0) & (qa[kx - 2] > qthr1)
    case_1 = mask_psa & (ktop1 < kx) & (ktop2 < kx)
    case_2 = mask_psa & (ktop1 < kx) & ~(ktop2 < kx) & lqthr
    iptop = np.where(case_1 | case_2, ktop1, iptop)
    qdif = np.where(case_1, np.maximum(qa[kx - 1] - qthr0, (mse0 - msthr) * rlhc), qdif)
    qdif = np.where(case_2, qa[kx - 1] - qthr0, qdif)
    return iptop, qdif


def get_convection_tendencies(state, data, params, forcing, geometry, rec=None):
    """get_convection_tendencies (convection.py:99-237)."""
    dt_ = state.temperature.dtype
    se = CP * state.temperature + state.geopotential
    qa = state.specific_humidity
    qsat = data.humidity.qsat
    kx, ix, il = se.shape
    psa = state.normalized_surface_pressure
    pc = params.convection
    dfse = np.zeros((kx, ix, il), dt_)
    dfqa = np.zeros((kx, ix, il), dt_)
    entr = np.maximum(0.0, geometry.fsg[1:kx - 1] - 0.5) ** 2.0
    sentr = np.sum(entr)
    entr = entr * (pc.entmax / sentr)
    fqmax = 5.0
    fm0 = P0 * geometry.dhs[-1] / (GRAV * pc.trcnv * 3600.0)
    rdps = 2.0 / (1.0 - pc.psmin)
    iptop, qdif = diagnose_convection(psa, se, qa, qsat, params, forcing, geometry, rec)
    mask = iptop < kx
    k = kx - 1
    qmax = np.maximum(1.01 * qa[-1], qsat[-1])

    def interp(tr):
        return tr[:-1] + geometry.wvi[:-1, 1, None, None] * np.diff(tr, axis=0)

    sb3 = np.zeros((kx, ix, il), dt_)
    sb3[1:] = interp(se)
    qb3 = np.zeros((kx, ix, il), dt_)
    qb3[1:] = interp(qa)
    sb = sb3[k]
    qb = np.minimum(qb3, qa)[k]
    with np.errstate(all="ignore"):
        fpsa = psa * np.minimum(1.0, (psa - pc.psmin) * rdps)
        fmass = fm0 * fpsa * np.minimum(fqmax, qdif / (qmax - qb))
    cbmf = mask * fmass
    fus, fuq = fmass * se[k], fmass * qmax
    fds, fdq = fmass * sb, fmass * qb
    dfse[k] = fds - fus
    dfqa[k] = fdq - fuq
    ar = np.arange(kx)[:, None, None]
    loop_mask = (kx - 2 >= ar) & (ar >= iptop)
    en = np.zeros((kx, ix, il), dt_)
    en[1:-1] = entr[:, None, None] * psa * cbmf
    enmass = loop_mask * en

    def rcum(x):
        # reverse cumulative sum, accumulated from the surface upwards
        out = np.empty_like(x)
        acc = np.zeros_like(x[0])
        for kk in range(x.shape[0] - 1, -1, -1):
            acc = acc + x[kk]
            out[kk] = acc
        return out

    fmass3 = fmass + rcum(enmass * 1)
    fus3 = fus + rcum(enmass * se)
    fuq3 = fuq + rcum(enmass * qa)
    fds3 = fmass3 * sb3
    fds3[-1] = fds
    fdq3 = fmass3 * qb3
    fdq3[-1] = fdq
    dfse[:-1] = loop_mask[:-1] * np.diff(fus3 - fds3, axis=0)
    dfqa[:-1] = loop_mask[:-1] * np.diff(fuq3 - fdq3, axis=0)
    delq = loop_mask * (pc.rhil * qsat - qa)
    _rec(rec, np.where(loop_mask, pc.rhil * qsat, 1.0), np.where(loop_mask, qa, 0.0))
    fsq = (delq > 0.0) * pc.smf * cbmf * delq
    dfqa = dfqa + fsq
    dfqa[-1] = dfqa[-1] + (-np.sum(fsq, axis=0))

    def pad(a):
        return np.concatenate([a, np.zeros((2,) + a.shape[1:], a.dtype)], axis=0)

    def at(a, idx):
        return np.take_along_axis(a, idx[None], axis=0)[0]

    fmass_t, fus_t, fuq_t, fds_t, fdq_t = (at(pad(f), iptop) for f in
                                           (fmass3, fus3, fuq3, fds3, fdq3))
    kt = iptop - 1
    qsatb = at(pad(interp(qsat)), kt)
    precnv = np.maximum(fuq_t - fmass_t * qsatb, 0.0)
    # top-layer scatter: JAX drops updates whose level index is out of range (kt == kx)
    ii, jj = np.meshgrid(np.arange(ix), np.arange(il), indexing="ij")
    ok = kt < kx
    dfse[kt[ok], ii[ok], jj[ok]] = (fus_t - fds_t + ALHC * precnv)[ok]
    dfqa[kt[ok], ii[ok], jj[ok]] = (fuq_t - fdq_t - precnv)[ok]
    with np.errstate(all="ignore"):
        rps = 1 / psa
    ttend = dfse.copy()
    ttend[1:] = dfse[1:] * rps * geometry.grdscp[1:, None, None]
    qtend = dfqa.copy()
    qtend[1:] = dfqa[1:] * rps * geometry.grdsig[1:, None, None]
    data = dcopy(data)
    data.convection.se = se
    data.convection.iptop = iptop
    data.convection.cbmf = cbmf
    data.convection.precnv = precnv
    tend = zero_tendency((kx, ix, il), dt_)
    tend.temperature = ttend
    tend.specific_humidity = qtend
    return tend, data


# ---------------------------------------------------------------------------------------------
# large_scale_condensation.py
# ---------------------------------------------------------------------------------------------
def get_large_scale_condensation_tendencies(state, data, params, forcing, geometry, rec=None):
    """get_large_scale_condensation_tendencies (large_scale_condensation.py:14-86)."""
    qa = state.specific_humidity
    dt_ = qa.dtype
    kx, ix, il = qa.shape
    qsat = data.humidity.qsat
    pc = params.condensation
    dtlsc = np.zeros_like(qa)
    dqlsc = np.zeros_like(qa)
    qsmax = 10.0
    rtlsc = 1.0 / (pc.trlsc * 3600.0)
    tfact = ALHC / CP
    prg = P0 / GRAV
    psa = state.normalized_surface_pressure
    psa2 = psa ** 2.0
    sig2 = geometry.fsg ** 2.0
    rhref = pc.rhlsc + pc.drhlsc * (sig2 - 1.0)
    rhref = np.maximum(rhref, pc.rhblsc)
    dqmax = qsmax * sig2 * rtlsc
    dqa = rhref[:, None, None] * qsat - qa
    _rec(rec, (rhref[:, None, None] * qsat)[1:], qa[1:])
    neg = dqa < 0
    dqlsc[1:] = np.where(neg[1:], dqa[1:] * rtlsc, 0.0)
    dtlsc[1:] = np.where(neg[1:], tfact * np.minimum(-dqlsc[1:], dqmax[1:, None, None] * psa2), 0.0)
    iptop = np.minimum(np.argmin(dqa[1:] >= 0, axis=0) + 1, data.convection.iptop)
    pfact = geometry.dhs * prg
    precls = 0.0 - np.sum(pfact[1:, None, None] * dqlsc[1:], axis=0)
    precls = precls * psa
    data = dcopy(data)
    data.condensation.precls = precls
    data.convection.iptop = iptop
    tend = zero_tendency((kx, ix, il), dt_)
    tend.temperature = dtlsc
    tend.specific_humidity = dqlsc
    return tend, data


# ---------------------------------------------------------------------------------------------
# shortwave_radiation.py (+ forcing.py set_forcing)
# ---------------------------------------------------------------------------------------------
def solar(tyear, csol=4.0 * SOLC, geometry=None, dtype=np.float32):
    """solar (shortwave_radiation.py:406-452): daily-mean TOA insolation per latitude."""
    tyear = dtype(tyear)
    pigr = 2.0 * np.arcsin(dtype(1.0))
    alpha = 2.0 * pigr * tyear
    ca1 = np.cos(alpha)
    sa1 = np.sin(alpha)
    ca2 = ca1 * ca1 - sa1 * sa1
    sa2 = 2.0 * sa1 * ca1
    ca3 = ca1 * ca2 - sa1 * sa2
    sa3 = sa1 * ca2 + sa2 * ca1
    decl = (0.006918 - 0.399912 * ca1 + 0.070257 * sa1 - 0.006758 * ca2 + 0.000907 * sa2
            - 0.002697 * ca3 + 0.001480 * sa3)
    fdis = 1.000110 + 0.034221 * ca1 + 0.001280 * sa1 + 0.000719 * ca2 + 0.000077 * sa2
    cdecl = np.cos(decl)
    sdecl = np.sin(decl)
    tdecl = sdecl / cdecl
    csolp = dtype(csol) / pigr
    ch0 = np.clip(-tdecl * geometry.sia / geometry.coa, dtype(-1 + EPSILON), dtype(1 - EPSILON))
    h0 = np.arccos(ch0)
    sh0 = np.sin(h0)
    return csolp * fdis * (h0 * geometry.sia * sdecl + sh0 * geometry.coa * cdecl)


def get_zonal_average_fields(state, data, forcing, geometry):
    """get_zonal_average_fields (shortwave_radiation.py:220-296)."""
    kx, ix, il = state.temperature.shape
    dtype = state.temperature.dtype.type
    tyear = dtype(data.date.tyear)
    asin1 = np.arcsin(dtype(1.0))
    alpha = 4.0 * asin1 * (tyear + 10.0 / 365.0)
    coz1 = np.maximum(0.0, np.cos(alpha - 0.0))
    coz2 = 1.8
    rzen = -np.cos(alpha) * 23.45 * asin1 / 90.0
    fs0 = 6.0
    topsr = solar(tyear, 4 * SOLC, geometry, dtype)
    sia, coa = geometry.sia, geometry.coa
    flat2 = 1.5 * sia ** 2 - 0.5
    fsol = topsr
    ozupp = 0.5 * EPSSW
    ozone = 0.4 * EPSSW * (1.0 + coz1 * sia + coz2 * flat2)
    base = 1.0 - (coa * np.cos(rzen) + sia * np.sin(rzen))
    zenit = 1.0 + 1.0 * (base * base)
    ozupp = fsol * ozupp * zenit
    ozone = fsol * ozone * zenit
    stratz = np.maximum(fs0 - fsol, 0.0)
    data = dcopy(data)
    b = lambda f: np.broadcast_to(np.asarray(f, dtype), (ix, il)).copy()
    data.shortwave_rad.fsol = b(fsol)
    data.shortwave_rad.ozupp = b(ozupp)
    data.shortwave_rad.ozone = b(ozone)
    data.shortwave_rad.zenit = b(zenit)
    data.shortwave_rad.stratz = b(stratz)
    return data


def set_forcing(state, data, params, forcing, geometry, rec=None):
    """set_forcing (physics/speedy/forcing.py:11-39)."""
    data = get_zonal_average_fields(state, data, forcing, geometry)
    dtype = state.temperature.dtype.type
    tyear = dtype(data.date.tyear)
    model_year = data.date.model_year
    fmask = geometry.fmask
    mr = params.mod_radcon
    snowc = np.minimum(1.0, forcing.snowc_am)
    alb_l = forcing.alb0 + snowc * (mr.albsn - forcing.alb0)
    alb_s = mr.albsea + forcing.sice_am * (mr.albice - mr.albsea)
    albsfc = alb_s + fmask * (alb_l - alb_s)
    iyear_ref = params.forcing.co2_year_ref
    inc = 1.0 if params.forcing.increase_co2 else 0.0
    ablco2 = ABLCO2_REF * exp_(inc * DEL_CO2 * (dtype(model_year) + tyear - iyear_ref))
    data.mod_radcon.snowc = snowc
    data.mod_radcon.alb_l = alb_l
    data.mod_radcon.alb_s = alb_s
    data.mod_radcon.albsfc = albsfc
    data.mod_radcon.ablco2 = dtype(ablco2)
    return None, data


def clouds(state, data, params, forcing, geometry, rec=None):
    """clouds (shortwave_radiation.py:313-404)."""
    se = data.convection.se
    phig = state.geopotential
    with np.errstate(all="ignore"):
        gse = (se[-2] - se[-1]) / (phig[-2] - phig[-1])
    rh = data.humidity.rh
    conv = data.convection
    kx = state.temperature.shape[0]
    ps = params.shortwave_radiation
    nl1 = kx - 2
    nlp = kx
    rrcl = 1.0 / (ps.rhcl2 - ps.rhcl1)
    _rec(rec, rh[nl1], ps.rhcl1)
    mask = rh[nl1] > ps.rhcl1
    cloudc = np.where(mask, rh[nl1] - ps.rhcl1, 0.0)
    icltop = np.where(mask, nl1, nlp)
    drh = rh[2:kx - 2] - ps.rhcl1
    _rec(rec, rh[2:kx - 2], (cloudc + ps.rhcl1)[None])  # drh > cloudc, on the scale of rh
    _rec(rec, state.specific_humidity[2:kx - 2], ps.qacl)
    m = (drh > cloudc) & (state.specific_humidity[2:kx - 2] > ps.qacl)
    cloudc_update = np.where(m, drh, cloudc)
    cloudc = np.max(cloudc_update, axis=0)
    kidx = np.arange(2, kx - 2)
    icltop_update = np.where(m, kidx[:, None, None], icltop)
    icltop = np.where(cloudc == cloudc_update, icltop_update, icltop).max(axis=0)
    with np.errstate(all="ignore"):
        pr1 = np.minimum(ps.pmaxcl, 86.4 * (conv.precnv + data.condensation.precls))
        cloudc = np.minimum(1.0, ps.wpcl * np.sqrt(np.maximum(EPSILON, pr1))
                            + np.minimum(1.0, cloudc * rrcl) ** 2.0)
    cloudc = np.where(np.isnan(cloudc), 1.0, cloudc)
    icltop = np.minimum(conv.iptop, icltop)
    qcloud = state.specific_humidity[nl1]
    clfact = 1.2
    rgse = 1.0 / (ps.gse_s1 - ps.gse_s0)
    fstab = np.clip(rgse * (gse - ps.gse_s0), 0.0, 1.0)
    clstr = fstab * np.maximum(ps.clsmax - clfact * cloudc, 0.0)
    clstrl = np.maximum(clstr, ps.clsminl) * rh[kx - 1]
    clstr = clstr + geometry.fmask * (clstrl - clstr)
    data = dcopy(data)
    sw = data.shortwave_rad
    sw.gse, sw.icltop, sw.cloudc, sw.cloudstr, sw.qcloud = gse, icltop, cloudc, clstr, qcloud
    return None, data


def get_clouds(state, data, params, forcing, geometry, rec=None):
    """get_clouds (shortwave_radiation.py:298-311); clouds never produce tendencies."""
    return clouds(state, data, params, forcing, geometry, rec)


def cloud_top_level_set(icltop, kx):
    """The level set S of shortwave_radiation.py:64-68.

    ``tau2.at[clip(icltop), :, :, 2].set(where(mask, albcl*cloudc, ...))`` indexes with a 2-D
    integer array and two slices, so under NumPy/JAX advanced-indexing rules it writes the whole
    ``(ix, il)`` plane ``where(mask, albcl*cloudc, 0)`` into every level that is *any* column's
    clipped ``icltop``.  Returns the boolean membership vector of length ``kx``.
    """
    s = np.zeros(kx, bool)
    s[np.unique(np.clip(icltop, 0, kx - 1))] = True
    return s


def shortwave_rad_fluxes(state, data, params, forcing, geometry, rec=None,
                         literal_scatter=False):
    """shortwave_rad_fluxes (shortwave_radiation.py:27-217).

    ``literal_scatter=True`` evaluates lines 62-68 with the reference's own advanced-indexing
    expression (an ``(ix, il, ix, il)`` temporary; small grids only); the default uses the
    equivalent level-set form.
    """
    kx, ix, il = state.temperature.shape
    dt_ = state.temperature.dtype
    dhs, fsg = geometry.dhs, geometry.fsg
    psa = state.normalized_surface_pressure
    qa = state.specific_humidity
    sw = data.shortwave_rad
    icltop, cloudc, clstr = sw.icltop, sw.cloudc, sw.cloudstr
    albsfc = data.mod_radcon.albsfc
    ps = params.shortwave_radiation
    nl1 = kx - 1
    fband2 = 0.05
    fband1 = 1.0 - fband2
    tau2 = np.zeros((kx, ix, il, 4), dt_)
    mask = icltop < kx
    clamped = np.clip(icltop, 0, kx - 1).astype(int)
    if literal_scatter:
        vals = np.where(mask, ps.albcl * cloudc, tau2[clamped, :, :, 2])
        tau2[clamped, :, :, 2] = vals
    else:
        plane = np.where(mask, ps.albcl * cloudc, 0.0).astype(dt_)
        for lev in np.nonzero(cloud_top_level_set(icltop, kx))[0]:
            tau2[lev, :, :, 2] = plane
    tau2[kx - 1, :, :, 2] = ps.albcls * clstr
    psaz = psa * sw.zenit
    acloud = cloudc * np.minimum(ps.abscl1 * sw.qcloud, ps.abscl2)
    tau2[0, :, :, 0] = exp_(-psaz * dhs[0] * ps.absdry)
    abs1 = ps.absdry + ps.absaer * fsg[1:nl1] ** 2
    cloudy = np.arange(1, nl1)[:, None, None] >= icltop
    tau2[1:nl1, :, :, 0] = exp_(-psaz * dhs[1:nl1, None, None] * (
        abs1[:, None, None] + ps.abswv1 * qa[1:nl1] + cloudy * acloud))
    abs1 = ps.absdry + ps.absaer * fsg[kx - 1] ** 2
    tau2[kx - 1, :, :, 0] = exp_(-psaz * dhs[kx - 1] * (abs1 + ps.abswv1 * qa[kx - 1]))
    tau2[1:kx, :, :, 1] = exp_(-psaz * dhs[1:kx, None, None] * ps.abswv2 * qa[1:kx])
    dfabs = np.zeros((kx, ix, il), dt_)
    ftop = sw.fsol
    flux_1 = np.zeros((kx, ix, il), dt_)
    flux_2 = np.zeros((kx, ix, il), dt_)
    flux_1[0] = sw.fsol * fband1
    flux_2[0] = sw.fsol * fband2
    dfabs[0] = flux_1[0]
    flux_1[0] = tau2[0, :, :, 0] * (flux_1[0] - sw.ozupp * psa)
    dfabs[0] = dfabs[0] + (-flux_1[0])
    flux_1[1] = flux_1[0]
    dfabs[1] = flux_1[1]
    flux_1[1] = tau2[1, :, :, 0] * (flux_1[1] - sw.ozone * psa)
    dfabs[1] = dfabs[1] + (-flux_1[1])
    for k in range(2, kx):
        flux_1[k] = flux_1[k - 1] * tau2[k, :, :, 0] * (1 - tau2[k, :, :, 2])
    dfabs[2:kx] = flux_1[1:kx - 1] * (1 - tau2[2:kx, :, :, 2]) * (1 - tau2[2:kx, :, :, 0])
    tau2[2:kx, :, :, 2] = tau2[2:kx, :, :, 2] * flux_1[1:kx - 1]
    flux_2[1] = flux_2[0]
    carry = flux_2[1]
    for k in range(1, kx):
        carry = carry * tau2[k, :, :, 1]
        flux_2[k] = carry
    dfabs[1:kx] = dfabs[1:kx] + flux_2[:kx - 1] * (1 - tau2[1:kx, :, :, 1])
    rsds = flux_1[kx - 1] + flux_2[kx - 1]
    flux_1[kx - 1] = flux_1[kx - 1] * albsfc
    rsns = rsds - flux_1[kx - 1]
    carry = flux_1[-1]
    up = np.zeros((kx - 1, ix, il), dt_)
    for k in range(kx - 1, 0, -1):
        carry = carry * tau2[k, :, :, 0] + tau2[k, :, :, 2]
        up[k - 1] = carry
    flux_1[:-1] = up
    dfabs = dfabs + flux_1 * (1 - tau2[:, :, :, 0])
    flux_1[1:] = flux_1[:-1].copy()
    flux_1[0] = tau2[0, :, :, 0] * flux_1[0] + tau2[0, :, :, 2]
    ftop = ftop - flux_1[0]
    ablco2 = data.mod_radcon.ablco2
    absorptivity = np.stack([ps.ablwin * np.ones_like(qa), ablco2 * np.ones_like(qa),
                             ps.ablwv1 * qa, ps.ablwv2 * qa], axis=-1).astype(dt_)
    absorptivity[0, :, :, 2:] = 0
    acloud1 = cloudc * ps.ablcl1
    acloud2 = cloudc * ps.ablcl2
    absorptivity[2:kx - 1, :, :, 0] = absorptivity[2:kx - 1, :, :, 0] + np.where(
        np.arange(2, kx - 1)[:, None, None] > icltop, acloud1, acloud2)
    absorptivity[2:kx - 1, :, :, 2:] = np.maximum(absorptivity[2:kx - 1, :, :, 2:],
                                                  acloud2[None, :, :, None])
    tau2 = exp_(-absorptivity * psa[:, :, None] * dhs[:, None, None, None])
    eps1 = params.mod_radcon.epslw / (dhs[0] + dhs[1])
    stratc = np.zeros((ix, il, 2), dt_)
    stratc[:, :, 0] = sw.stratz * psa
    stratc[:, :, 1] = eps1 * psa
    flux = data.mod_radcon.flux.copy()
    flux[:, :, 0] = flux_1[0]
    flux[:, :, 1] = flux_2[kx - 1]
    data = dcopy(data)
    data.mod_radcon.tau2, data.mod_radcon.stratc, data.mod_radcon.flux = tau2, stratc, flux
    s = data.shortwave_rad
    s.rsns, s.ftop, s.dfabs, s.rsds = rsns, ftop, dfabs, rsds
    ttend = dfabs * geometry.grdscp[:, None, None] / psa
    tend = zero_tendency((kx, ix, il), dt_)
    tend.temperature = ttend
    return tend, data


def get_shortwave_rad_fluxes(state, data, params, forcing, geometry, rec=None):
    """get_shortwave_rad_fluxes (shortwave_radiation.py:12-25): tendencies gated by nstrad."""
    tend, data = shortwave_rad_fluxes(state, data, params, forcing, geometry, rec)
    if not data.shortwave_rad.compute_shortwave:
        tend = zero_tendency(state.temperature.shape, state.temperature.dtype)
    return tend, data


# ---------------------------------------------------------------------------------------------
# longwave_radiation.py
# ---------------------------------------------------------------------------------------------
def radset(temp, epslw):
    """radset (longwave_radiation.py:204-226): energy fraction per LW band."""
    jtemp = np.clip(temp, 200, 320)
    f1 = 0.148 - 3.0e-6 * (jtemp - 247) ** 2
    f2 = 0.356 - 5.2e-6 * (jtemp - 282) ** 2
    f3 = 0.314 + 1.0e-5 * (jtemp - 315) ** 2
    f0 = 1.0 - (((np.zeros_like(jtemp) + f1) + f2) + f3)
    return (1.0 - epslw) * np.stack((f0, f1, f2, f3), axis=-1)


def get_downward_longwave_rad_fluxes(state, data, params, forcing, geometry, rec=None):
    """get_downward_longwave_rad_fluxes (longwave_radiation.py:13-117)."""
    kx, ix, il = state.temperature.shape
    dt_ = state.temperature.dtype
    ta = state.temperature
    st4a = data.mod_radcon.st4a.copy()
    tau2 = data.mod_radcon.tau2
    mr = params.mod_radcon
    nl1 = kx - 1
    st4a[:nl1, :, :, 0] = ta[:nl1] + geometry.wvi[:nl1, 1, None, None] * (ta[1:nl1 + 1] - ta[:nl1])
    st4a[0, :, :, 1] = 0.75 * ta[0] + 0.25 * st4a[0, :, :, 0]
    st4a[1, :, :, 1] = 0.50 * ta[1] + 0.25 * (st4a[0, :, :, 0] + st4a[1, :, :, 0])
    st4a[2:nl1, :, :, 1] = 0.5 * 1 * np.maximum(st4a[2:nl1, :, :, 0] - st4a[1:nl1 - 1, :, :, 0], 0.0)
    st4a[kx - 1, :, :, 1] = 1 * np.maximum(ta[kx - 1] - st4a[nl1 - 1, :, :, 0], 0.0)
    st4a[:2, :, :, 0] = SBC * st4a[:2, :, :, 1] ** 4.0
    st4a[:2, :, :, 1] = 0.0
    st3a = SBC * ta[2:kx] ** 3.0
    st4a[2:kx, :, :, 0] = st3a * ta[2:kx]
    st4a[2:kx, :, :, 1] = 4.0 * st3a * st4a[2:kx, :, :, 1]
    dfabs = np.zeros((kx, ix, il), dt_)
    emis = 1 - tau2
    brad = radset(ta, mr.epslw) * (st4a[:, :, :, 0, None] + emis * st4a[:, :, :, 1, None])
    emis_brad = emis * brad
    flux = emis_brad[0].copy()
    flux[:, :, 2:4] = 0.0
    dfabs[0] = dfabs[0] + (-np.sum(flux, axis=-1))
    f3d = np.zeros((kx, ix, il, 4), dt_)
    f3d[0] = flux
    for k in range(1, kx):
        flux = tau2[k] * flux + emis_brad[k]
        f3d[k] = flux
    dfabs[1:] = dfabs[1:] + (-np.diff(np.sum(f3d, axis=-1), axis=0))
    rlds = np.sum(mr.emisfc * flux, axis=-1)
    corlw = mr.epslw * mr.emisfc * st4a[kx - 1, :, :, 0]
    dfabs[-1] = dfabs[-1] + (-corlw)
    rlds = rlds + corlw
    data = dcopy(data)
    data.surface_flux.rlds = rlds
    data.longwave_rad.dfabs = dfabs
    data.mod_radcon.st4a = st4a
    return None, data


def get_upward_longwave_rad_fluxes(state, data, params, forcing, geometry, rec=None):
    """get_upward_longwave_rad_fluxes (longwave_radiation.py:119-202)."""
    kx, ix, il = state.temperature.shape
    dt_ = state.temperature.dtype
    ta = state.temperature
    dfabs = data.longwave_rad.dfabs.copy()
    rlds = data.surface_flux.rlds
    st4a = data.mod_radcon.st4a
    flux = data.mod_radcon.flux
    tau2 = data.mod_radcon.tau2
    stratc = data.mod_radcon.stratc
    mr = params.mod_radcon
    rlus = data.surface_flux.rlus[:, :, 2]
    ts = data.surface_flux.tsfc
    refsfc = 1.0 - mr.emisfc
    epslw = mr.epslw
    fsfc = rlus - rlds
    flux = radset(ts, epslw) * rlus[:, :, None] + refsfc * flux
    dfabs[-1] = dfabs[-1] + epslw * rlus
    emis = 1.0 - tau2
    brad = radset(ta, epslw) * (st4a[:, :, :, 0, None] - emis * st4a[:, :, :, 1, None])
    emis_brad = emis * brad
    f3d = np.zeros((kx, ix, il, 4), dt_)
    f3d[-1] = flux
    for k in range(kx - 1, 0, -1):
        flux = tau2[k] * flux + emis_brad[k]
        f3d[k - 1] = flux
    flux = f3d[0].copy()
    dfabs[1:] = dfabs[1:] + np.diff(np.sum(f3d, axis=-1), axis=0)
    flux[:, :, :2] = (tau2[0] * flux + emis_brad[0])[:, :, :2]
    dfabs[0] = dfabs[0] + np.sum((f3d[0] - flux)[:, :, :2], axis=-1)
    corlw1 = geometry.dhs[0] * stratc[:, :, 1] * st4a[0, :, :, 0] + stratc[:, :, 0]
    corlw2 = geometry.dhs[1] * stratc[:, :, 1] * st4a[1, :, :, 0]
    dfabs[0] = dfabs[0] + (-corlw1)
    dfabs[1] = dfabs[1] + (-corlw2)
    ftop = corlw1 + corlw2
    ftop = ftop + np.sum(flux, axis=-1)
    data = dcopy(data)
    data.surface_flux.rlns = fsfc
    data.longwave_rad.ftop = ftop
    data.longwave_rad.dfabs = dfabs
    data.mod_radcon.flux = flux
    tend = zero_tendency((kx, ix, il), dt_)
    tend.temperature = dfabs * geometry.grdscp[:, None, None] / state.normalized_surface_pressure
    return tend, data


# ---------------------------------------------------------------------------------------------
# surface_flux.py
# ---------------------------------------------------------------------------------------------
def get_orog_land_sfc_drag(phis0, hdrag):
    """get_orog_land_sfc_drag (surface_flux.py:302-315)."""
    rhdrag = 1 / (GRAV * hdrag)
    return 1.0 + rhdrag * (1.0 - exp_(-np.maximum(phis0, 0.0) * rhdrag))


def get_surface_fluxes(state, data, params, forcing, geometry, rec=None):
    """get_surface_fluxes (surface_flux.py:15-300)."""
    stl_am = forcing.stl_am
    sst = forcing.sea_surface_temperature
    kx, ix, il = state.temperature.shape
    dt_ = state.temperature.dtype
    psa = state.normalized_surface_pressure
    ua, va, ta, qa, phi = (state.u_wind, state.v_wind, state.temperature,
                           state.specific_humidity, state.geopotential)
    fmask = geometry.fmask
    rsds = data.shortwave_rad.rsds
    rlds = data.surface_flux.rlds
    rh = data.humidity.rh
    phi0 = geometry.orog * GRAV
    snowc, alb_l, alb_s = data.mod_radcon.snowc, data.mod_radcon.alb_l, data.mod_radcon.alb_s
    sf, mr = params.surface_flux, params.mod_radcon
    esbc = mr.emisfc * SBC
    ghum0 = 1.0 - sf.fhum0
    z = lambda *s: np.zeros((ix, il) + s, dt_)
    ustr, vstr, shf, evap, rlus = z(3), z(3), z(3), z(3), z(3)
    hfluxn, t1, q1, t2, qsat0, denvvs = z(2), z(2), z(2), z(2), z(2), z(3)
    u0 = sf.fwind0 * ua[kx - 1]
    v0 = sf.fwind0 * va[kx - 1]
    tskin = np.zeros_like(stl_am)
    astab = 0.5 if sf.lscasym else 1.0
    rdth = sf.fstab / sf.dtheta
    if forcing.lfluxland:
        rcp = 1.0 / CP
        nl1 = kx - 1
        gtemp0 = 1.0 - sf.ftemp0
        dt1 = geometry.wvi[kx - 1, 1] * (ta[kx - 1] - ta[nl1 - 1])
        t1[:, :, 0] = t1[:, :, 0] + (ta[kx - 1] + dt1)
        t1[:, :, 1] = t1[:, :, 0] - phi0 * dt1 / (RGAS * 288.0 * geometry.sigl[kx - 1])
        t2[:, :, 1] = ta[kx - 1] + rcp * phi[kx - 1]
        t2[:, :, 0] = t2[:, :, 1] - rcp * phi0
        _rec(rec, ta[kx - 1], ta[nl1 - 1])
        t1 = np.where((ta[kx - 1] > ta[nl1 - 1])[:, :, None], sf.ftemp0 * t1 + gtemp0 * t2,
                      ta[kx - 1][:, :, None])
        t0 = t1[:, :, 1] + fmask * (t1[:, :, 0] - t1[:, :, 1])
        with np.errstate(all="ignore"):
            denvvs[:, :, 0] = (P0 * psa / (RGAS * t0)) * np.sqrt(u0 * u0 + v0 * v0 + sf.vgust * sf.vgust)
        tskin = stl_am + sf.ctday * np.sqrt(geometry.coa) * rsds * (1.0 - alb_l) * psa
        _rec(rec, tskin, t2[:, :, 0])
        dthl = np.where(tskin > t2[:, :, 0], np.minimum(sf.dtheta, tskin - t2[:, :, 0]),
                        np.maximum(-sf.dtheta, astab * (tskin - t2[:, :, 0])))
        denvvs[:, :, 1] = denvvs[:, :, 0] * (1.0 + dthl * rdth)
        forog = get_orog_land_sfc_drag(geometry.phis0, sf.hdrag)
        cdldv = sf.cdl * denvvs[:, :, 0] * forog
        ustr[:, :, 0] = -cdldv * ua[kx - 1]
        vstr[:, :, 0] = -cdldv * va[kx - 1]
        chlcp = sf.chl * CP
        shf[:, :, 0] = chlcp * denvvs[:, :, 1] * (tskin - t1[:, :, 0])

        def evap_q1(idx):
            if sf.fhum0 > 0.0:
                q1v, qs = rel_hum_to_spec_hum(t1[:, :, idx], psa, 1.0, rh[kx - 1])
                q1[:, :, idx] = sf.fhum0 * q1v + ghum0 * qa[kx - 1]
                qsat0[:, :, idx] = qs
            else:
                q1[:, :, idx] = qa[kx - 1]

        evap_q1(0)
        qsat0[:, :, 0] = get_qsat(tskin, psa, 1.0, rec)
        evap[:, :, 0] = sf.chl * denvvs[:, :, 1] * np.maximum(
            0.0, forcing.soilw_am * qsat0[:, :, 0] - q1[:, :, 0])
        tsk3 = tskin ** 3.0
        drls = 4.0 * esbc * tsk3
        rlus[:, :, 0] = esbc * tsk3 * tskin
        hfluxn[:, :, 0] = rsds * (1.0 - alb_l) + rlds - (rlus[:, :, 0] + shf[:, :, 0] + (ALHC * evap[:, :, 0]))
        if sf.lskineb:
            clamb = sf.clambda + (snowc * (sf.clambsn - sf.clambda))
            hfluxn[:, :, 0] = hfluxn[:, :, 0] - (clamb * (tskin - stl_am))
            dtskin = tskin + 1.0
            qsat0[:, :, 1] = get_qsat(dtskin, psa, 1.0, rec)
            # evap > 0: the sign of soilw qsat0 - q1 under the max(0, .) above
            _rec(rec, forcing.soilw_am * qsat0[:, :, 0], q1[:, :, 0])
            qsat0[:, :, 1] = np.where(evap[:, :, 0] > 0.0,
                                      forcing.soilw_am * (qsat0[:, :, 1] - qsat0[:, :, 0]), 0.0)
            with np.errstate(all="ignore"):
                dtskin = hfluxn[:, :, 0] / (clamb + drls + (sf.chl * denvvs[:, :, 1] * (CP + (ALHC * qsat0[:, :, 1]))))
            tskin = tskin + dtskin
            shf[:, :, 0] = shf[:, :, 0] + chlcp * denvvs[:, :, 1] * dtskin
            evap[:, :, 0] = evap[:, :, 0] + sf.chl * denvvs[:, :, 1] * qsat0[:, :, 1] * dtskin
            rlus[:, :, 0] = rlus[:, :, 0] + drls * dtskin
            hfluxn[:, :, 0] = clamb * (tskin - stl_am)
        _rec(rec, sst, t2[:, :, 1])
        dths = np.where(sst > t2[:, :, 1], np.minimum(sf.dtheta, sst - t2[:, :, 1]),
                        np.maximum(-sf.dtheta, astab * (sst - t2[:, :, 1])))
        denvvs[:, :, 2] = denvvs[:, :, 0] * (1.0 + dths * rdth)
        evap_q1(1)
        cdsdv = sf.cds * denvvs[:, :, 2]
        ustr[:, :, 1] = -cdsdv * ua[kx - 1]
        vstr[:, :, 1] = -cdsdv * va[kx - 1]
    ks = 2
    shf[:, :, 1] = sf.chs * CP * denvvs[:, :, ks] * (sst - t1[:, :, 1])
    qsat0[:, :, 1] = get_qsat(sst, psa, 1.0, rec)
    evap[:, :, 1] = sf.chs * denvvs[:, :, ks] * (qsat0[:, :, 1] - q1[:, :, 1])
    rlus[:, :, 1] = esbc * (sst ** 4.0)
    hfluxn[:, :, 1] = rsds * (1.0 - alb_s) + rlds - rlus[:, :, 1] + shf[:, :, 1] + ALHC * evap[:, :, 1]
    wavg = lambda var: var[:, :, 1] + fmask * (var[:, :, 0] - var[:, :, 1])
    t0 = np.zeros_like(t1[:, :, 0])
    tsfc = np.zeros_like(stl_am)
    if forcing.lfluxland:
        for v in (ustr, vstr, shf, evap, rlus):
            v[:, :, 2] = wavg(v)
        t0 = wavg(t1)
        tsfc = sst + fmask * (stl_am - sst)
        tskin = sst + fmask * (tskin - sst)
    data = dcopy(data)
    s = data.surface_flux
    s.ustr, s.vstr, s.shf, s.evap, s.rlus = ustr, vstr, shf, evap, rlus
    s.hfluxn, s.tsfc, s.tskin, s.u0, s.v0, s.t0 = hfluxn, tsfc, tskin, u0, v0, t0
    with np.errstate(all="ignore"):
        rps = 1.0 / psa
    tend = zero_tendency((kx, ix, il), dt_)
    tend.u_wind[-1] = tend.u_wind[-1] + ustr[:, :, 2] * rps * geometry.grdsig[-1]
    tend.v_wind[-1] = tend.v_wind[-1] + vstr[:, :, 2] * rps * geometry.grdsig[-1]
    tend.temperature[-1] = tend.temperature[-1] + shf[:, :, 2] * rps * geometry.grdscp[-1]
    tend.specific_humidity[-1] = tend.specific_humidity[-1] + evap[:, :, 2] * rps * geometry.grdsig[-1]
    return tend, data


# ---------------------------------------------------------------------------------------------
# vertical_diffusion.py
# ---------------------------------------------------------------------------------------------
def get_vertical_diffusion_tend(state, data, params, forcing, geometry, rec=None):
    """get_vertical_diffusion_tend (vertical_diffusion.py:10-136)."""
    se = data.convection.se
    rh = data.humidity.rh
    qsat = data.humidity.qsat
    qa = state.specific_humidity
    phi = state.geopotential
    kx, ix, il = state.temperature.shape
    dt_ = state.temperature.dtype
    pv = params.vertical_diffusion
    hsg, fsg, dhs = geometry.hsg, geometry.fsg, geometry.dhs
    icnv = kx - data.convection.iptop - 1
    tt = np.zeros((kx, ix, il), dt_)
    qt = np.zeros((kx, ix, il), dt_)
    nl1 = kx - 1
    cshc = dhs[kx - 1] / 3600.0
    cvdi = (hsg[nl1] - hsg[1]) / ((nl1 - 1) * 3600.0)
    fshcq = cshc / pv.trshc
    fshcse = cshc / (pv.trshc * CP)
    fvdiq = cvdi / pv.trvdi
    fvdise = cvdi / (pv.trvds * CP)
    rsig = 1.0 / dhs
    rsig1 = np.zeros((kx,), dt_)
    rsig1[:-1] = 1.0 / (1.0 - hsg[1:-1])
    rsig1[-1] = 0.0
    drh0 = pv.rhgrad * (fsg[kx - 1] - fsg[nl1 - 1])
    fvdiq2 = fvdiq * hsg[nl1]
    dmse = se[kx - 1] - se[nl1 - 1] + ALHC * (qa[kx - 1] - qsat[nl1 - 1])
    drh = rh[kx - 1] - rh[nl1 - 1]
    # dmse >= 0, drh >= 0 and drh >= drh0, each between the quantities the differences cancel
    _rec(rec, se[kx - 1] + ALHC * qa[kx - 1], se[nl1 - 1] + ALHC * qsat[nl1 - 1])
    _rec(rec, rh[kx - 1], rh[nl1 - 1])
    _rec(rec, rh[kx - 1], rh[nl1 - 1] + drh0)
    fcnv = np.ones((ix, il), dt_)
    fcnv = np.where(np.logical_and(icnv > 0, dmse >= 0), pv.redshc, fcnv)
    fluxse = np.where(dmse >= 0.0, fcnv * fshcse * dmse, 0)
    tt[nl1 - 1] = np.where(dmse >= 0.0, fluxse * rsig[nl1 - 1], tt[nl1 - 1])
    tt[kx - 1] = np.where(dmse >= 0.0, -fluxse * rsig[kx - 1], tt[kx - 1])
    c1 = (dmse >= 0.0) & (drh >= 0.0)
    fq1 = np.where(c1, fcnv * fshcq * qsat[kx - 1] * drh, 0)
    qt[nl1 - 1] = np.where(c1, fq1 * rsig[nl1 - 1], qt[nl1 - 1])
    qt[kx - 1] = np.where(c1, -fq1 * rsig[kx - 1], qt[kx - 1])
    c2 = (dmse < 0.0) & (drh > drh0)
    fq2 = np.where(c2, fvdiq2 * qsat[nl1 - 1] * drh, 0)
    qt[nl1 - 1] = np.where(c2, fq2 * rsig[nl1 - 1], qt[nl1 - 1])
    qt[kx - 1] = np.where(c2, -fq2 * rsig[kx - 1], qt[kx - 1])
    kr = np.arange(2, kx - 2)
    cond = hsg[kr + 1] > 0.5
    drh0v = pv.rhgrad * (fsg[kr + 1] - fsg[kr])
    fvdiq2v = fvdiq * hsg[kr + 1]
    drhv = rh[kr + 1] - rh[kr]
    _rec(rec, rh[kr + 1], rh[kr] + drh0v[:, None, None])  # drhv >= drh0v, on the scale of rh
    fluxq = np.where((drhv >= drh0v[:, None, None]) & cond[:, None, None],
                     fvdiq2v[:, None, None] * qsat[kr] * drhv, 0)
    qt[kr] = qt[kr] + fluxq * rsig[kr][:, None, None]
    qt[kr + 1] = qt[kr + 1] + (-fluxq * rsig[kr + 1][:, None, None])
    se0 = se[1:] - pv.segrad * np.diff(phi, axis=0)
    _rec(rec, se[:nl1], se0)
    cnd = se[:nl1] < se0
    fse = np.where(cnd, fvdise * (se0 - se[:nl1]), 0)
    tt[:nl1] = tt[:nl1] + fse * rsig[:nl1, None, None]
    cum = np.cumsum(fse * rsig1[:nl1, None, None], axis=0)
    tt[1:] = tt[1:] + (-cum)
    tend = zero_tendency((kx, ix, il), dt_)
    tend.temperature = tt.astype(dt_)
    tend.specific_humidity = qt.astype(dt_)
    return tend, data


# ---------------------------------------------------------------------------------------------
# speedy_physics.py + physics_interface.py
# ---------------------------------------------------------------------------------------------
def set_physics_flags(state, data, params, forcing, geometry, rec=None):
    """set_physics_flags (speedy_physics.py:13-32)."""
    data = dcopy(data)
    data.shortwave_rad.compute_shortwave = bool(int(data.date.model_step) % NSTRAD == 0)
    return None, data


TERMS = [set_physics_flags, set_forcing, spec_hum_to_rel_hum, get_convection_tendencies,
         get_large_scale_condensation_tendencies, get_clouds, get_shortwave_rad_fluxes,
         get_downward_longwave_rad_fluxes, get_surface_fluxes,
         get_upward_longwave_rad_fluxes, get_vertical_diffusion_tend]


# ---------------------------------------------------------------------------------------------
# orographic_correction.py (the optional last term; commented out of the reference's term list
# at speedy_physics.py:65,79)
# ---------------------------------------------------------------------------------------------
GAMMA = 6.0     # physical_constants.py:24, reference lapse rate (K/km)
HSCALE = 7.5    # physical_constants.py:25
HSHUM = 2.5     # physical_constants.py:26
REFRH1 = 0.7    # physical_constants.py:27


def orographic_vertical_profiles(fsg):
    """compute_temperature_correction_vertical_profile / ..._humidity_... (orographic_correction.py
    :18-93): tcorv = fsg^(rgas gamma / (1000 g)) except level 0; qcorv = fsg^(hscale / hshum)
    except levels 0 and 1."""
    rgam = RGAS * GAMMA / (1000.0 * GRAV)
    qexp = HSCALE / HSHUM
    k = np.arange(fsg.shape[0])
    tcorv = np.where(k == 0, 0.0, fsg ** rgam).astype(fsg.dtype)
    qcorv = np.where(k < 2, 0.0, fsg ** qexp).astype(fsg.dtype)
    return tcorv, qcorv


def orographic_horizontal(phis0, fmask, stl, sst):
    """compute_temperature_correction_horizontal and compute_humidity_correction_horizontal
    (orographic_correction.py:96-174).  The reference's get_qsat with sig <= 0 divides by the
    first element of its pressure field (humidity.py:100-101); the caller passes ones there, so
    that is 1."""
    dt_ = phis0.dtype.type
    gamlat = GAMMA / (1000.0 * GRAV)
    tcorh = gamlat * phis0
    tsfc = fmask * stl + (1.0 - fmask) * sst
    tref = tsfc + tcorh
    pexp = 1000.0 * GRAV / (RGAS * GAMMA)
    with np.errstate(all="ignore"):
        psfc = (tsfc / tref) ** pexp

        def esat(ta):
            return np.where(ta >= 273.16, 6.108e-3 * exp_(17.269 * (ta - 273.16) / (ta - 35.86)),
                            6.108e-3 * exp_(21.875 * (ta - 273.16) / (ta - 7.66)))
        e_ref = esat(tref)
        qref = 622.0 * e_ref / (dt_(1.0) - 0.378 * e_ref)
        qsfc = get_qsat(tsfc, psfc, dt_(1.0))
    qcorh = REFRH1 * (qref - qsfc)
    return tcorh.astype(phis0.dtype), qcorh.astype(phis0.dtype)


def get_orographic_correction_tendencies(state, data, params, forcing, geometry, rec=None):
    """get_orographic_correction_tendencies (orographic_correction.py:177-247): the correction
    tcorh*tcorv (temperature) and qcorh*qcorv (humidity) spread over one model step."""
    tcorv, qcorv = orographic_vertical_profiles(geometry.fsg)
    tcorh, qcorh = orographic_horizontal(geometry.phis0, geometry.fmask, forcing.stl_am,
                                         forcing.sea_surface_temperature)
    dt = data.date.dt_seconds
    t = zero_tendency(state.temperature.shape, state.temperature.dtype)
    t.temperature = (tcorh[None] * tcorv[:, None, None]) / dt
    t.specific_humidity = (qcorh[None] * qcorv[:, None, None]) / dt
    return t, data


TERMS_OROGRAPHIC = TERMS + [get_orographic_correction_tendencies]


def forcing_day_slice(forcing, date):
    """tree_index_3d(forcing, date.model_day()) (speedy_physics.py:119-121, utils.py:104-108)."""
    day = model_day(date)
    f = dcopy(forcing)
    for k in ("alb0", "sice_am", "snowc_am", "soilw_am", "stl_am", "sea_surface_temperature"):
        a = getattr(f, k)
        if a.ndim > 2:
            setattr(f, k, a[:, :, day])
    return f


def compute_tendencies(state, forcing, geometry, date, params, rec=None, orographic=False):
    """SpeedyPhysics.compute_tendencies (speedy_physics.py:88-127).

    Tendencies are summed in float ``dtype`` in term order; ``orographic`` appends the
    orographic correction as the last term.
    """
    kx, ix, il = state.temperature.shape
    dt_ = state.temperature.dtype
    data = zeros_data((ix, il), kx, date, dt_)
    tend = zero_tendency((kx, ix, il), dt_)
    forcing_2d = forcing_day_slice(forcing, date)
    for term in (TERMS_OROGRAPHIC if orographic else TERMS):
        t, data = term(state, data, params, forcing_2d, geometry, rec)
        if t is not None:
            tend.u_wind = tend.u_wind + t.u_wind
            tend.v_wind = tend.v_wind + t.v_wind
            tend.temperature = tend.temperature + t.temperature
            tend.specific_humidity = tend.specific_humidity + t.specific_humidity
    return tend, data


def verify_state(state):
    """verify_state (physics_interface.py:305-319): negative humidity clamped to zero."""
    s = dcopy(state)
    s.specific_humidity = np.where(state.specific_humidity < 0.0, 0.0,
                                   state.specific_humidity).astype(state.specific_humidity.dtype)
    return s


def verify_tendencies(state, tend, time_step):
    """verify_tendencies (physics_interface.py:321-342), with the unclamped state."""
    t = dcopy(tend)
    q = state.specific_humidity
    dq = tend.specific_humidity
    t.specific_humidity = np.where(q + time_step * dq >= 0, dq, -q / time_step).astype(dq.dtype)
    return t


def physics_step(state, forcing, geometry, date, params, time_step=None, fuse_verify=True,
                 rec=None, orographic=False):
    """The physics part of get_physical_tendencies (physics_interface.py:371-376)."""
    if not fuse_verify:
        return compute_tendencies(state, forcing, geometry, date, params, rec, orographic)
    dt_ = state.temperature.dtype.type
    ts = dt_(date.dt_seconds if time_step is None else time_step)
    tend, data = compute_tendencies(verify_state(state), forcing, geometry, date, params, rec,
                                    orographic)
    return verify_tendencies(state, tend, ts), data


def cast_inputs(state, forcing, geometry, date, params, dtype):
    """Recast every float leaf to ``dtype`` (float64 for the x64 error report)."""
    def cast_ns(o):
        o = dcopy(o)
        for k, v in vars(o).items():
            if isinstance(v, np.ndarray) and v.dtype.kind == "f":
                setattr(o, k, v.astype(dtype))
            elif isinstance(v, (np.floating,)):
                setattr(o, k, dtype(v))
            elif isinstance(v, SimpleNamespace):
                setattr(o, k, cast_ns(v))
        return o
    return (cast_ns(state), cast_ns(forcing), cast_ns(geometry), cast_ns(date),
            cast_ns(params))
