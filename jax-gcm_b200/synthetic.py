"""Seeded synthetic SPEEDY columns with the shapes and value distributions of the benchmark
workloads (no dataset ships with the reference, so these stand in for real model states).

* ``config0_instance`` -- T31 aquaplanet: 96x48 Gaussian grid, 8 sigma levels, all ocean.
* ``land_instance``    -- the ensemble member generator: land fraction, orography, soil
  moisture, snow and sea ice over the config-0 atmosphere.
* ``ensemble_members`` -- the ragged ensemble 32xT21, 16xT31, 8xT42, 4xT85, 1xT170 (466,944
  columns), members alternating 8/16 levels inside each resolution group, T170 at 16.
* ``t425_instance``    -- 1280x640 columns at 16 levels with the ensemble's surface fields.

Everything is float32 in the reference layout: level fields ``[kx, ix, il]``, surface fields
``[ix, il]``, latitude tables ``[il]`` (south to north).  Geopotential is not part of the
workload description; it is built hydrostatically as ``phi_s + rgas*T*(-ln sigma)``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

GRAV = 9.81
CP = 1004.0
RGAS = 2.0 / 7.0 * CP
DAYS_YEAR = 365.2425

SIGMA_LAYER_BOUNDARIES = {
    7: [0.0, 0.14, 0.26, 0.42, 0.6, 0.77, 0.9, 1.0],
    8: [0.0, 0.05, 0.14, 0.26, 0.42, 0.6, 0.77, 0.9, 1.0],
    16: [k / 16.0 for k in range(17)],
}

# nodal shape (ix, il) of each spectral truncation (jcm/utils.py:12-23)
GRIDS = {21: (64, 32), 31: (96, 48), 42: (128, 64), 85: (256, 128), 106: (320, 160),
         119: (360, 180), 170: (512, 256), 213: (640, 320), 340: (1024, 512), 425: (1280, 640)}


def vertical_tables(kx):
    """Vertical sigma tables of a kx-level grid (geometry.py:62-85), float32."""
    f = np.float32
    hsg = np.asarray(SIGMA_LAYER_BOUNDARIES[kx], f)
    fsg = (hsg[1:] + hsg[:-1]) / f(2.0)
    dhs = np.diff(hsg)
    sigl = np.log(fsg)
    grdsig = f(GRAV) / (dhs * f(1e5))
    grdscp = grdsig / f(CP)
    wvi = np.zeros((kx, 2), f)
    wvi[:-1, 0] = f(1.0) / np.diff(sigl)
    wvi[:-1, 1] = (np.log(hsg[1:-1]) - sigl[:-1]) * wvi[:-1, 0]
    wvi[-1, 1] = (np.log(f(0.99)) - sigl[-1]) * wvi[-2, 0]
    return dict(hsg=hsg, fsg=fsg, dhs=dhs, sigl=sigl, grdsig=grdsig, grdscp=grdscp, wvi=wvi)


def qsat_f32(ta, ps, sig):
    """Saturation specific humidity in g/kg (the Tetens form of humidity.py:97-102)."""
    f = np.float32
    e = np.where(ta >= f(273.16), f(6.108e-3) * np.exp(f(17.269) * (ta - f(273.16)) / (ta - f(35.86))),
                 f(6.108e-3) * np.exp(f(21.875) * (ta - f(273.16)) / (ta - f(7.66))))
    return f(622.0) * e / (sig * ps - f(0.378) * e)


@dataclass
class Instance:
    """One grid (one ensemble member): state, forcing, geometry and date."""
    kx: int
    ix: int
    il: int
    u: np.ndarray
    v: np.ndarray
    t: np.ndarray
    q: np.ndarray
    phi: np.ndarray
    psa: np.ndarray
    sst: np.ndarray
    stl: np.ndarray
    soilw: np.ndarray
    snowc: np.ndarray
    sice: np.ndarray
    alb0: np.ndarray
    fmask: np.ndarray
    orog: np.ndarray
    phis0: np.ndarray
    lat: np.ndarray  # radians, float64
    sia: np.ndarray
    coa: np.ndarray
    vert: dict
    tyear: float = 80.0 / DAYS_YEAR
    model_year: int = 1950
    model_step: int = 0
    dt_seconds: float = 1800.0
    lfluxland: bool = True
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def columns(self):
        return self.ix * self.il

    STATE = ("u", "v", "t", "q", "phi")
    SURFACE = ("psa", "sst", "stl", "soilw", "snowc", "sice", "alb0", "fmask", "orog", "phis0")

    def oracle_args(self, params):
        """(state, forcing, geometry, date, params) in the oracle's containers (tests only)."""
        from oracle import speedy_oracle as O
        st = O.make_state((self.kx, self.ix, self.il), u_wind=self.u, v_wind=self.v,
                          temperature=self.t, specific_humidity=self.q, geopotential=self.phi,
                          normalized_surface_pressure=self.psa)
        fo = O.make_forcing((self.ix, self.il), lfluxland=self.lfluxland, alb0=self.alb0,
                            sice_am=self.sice, snowc_am=self.snowc, soilw_am=self.soilw,
                            stl_am=self.stl, sea_surface_temperature=self.sst)
        ge = O.make_geometry(self.ix, self.il, self.kx, lat=self.lat, orog=self.orog,
                             fmask=self.fmask, phis0=self.phis0)
        ge.sia, ge.coa = self.sia.copy(), self.coa.copy()
        da = O.make_date(self.tyear, self.model_year, self.model_step, self.dt_seconds)
        return st, fo, ge, da, params


def gaussian_latitudes(il):
    x, _ = np.polynomial.legendre.leggauss(il)
    return np.arcsin(x)


def _atmosphere(rng, kx, ix, il, lat, phis):
    f = np.float32
    vert = vertical_tables(kx)
    sig = vert["fsg"].astype(np.float64)[:, None, None]
    shape = (kx, ix, il)
    t = 288.0 - 6.5 * (-7.0 * np.log(sig)) + rng.normal(0.0, 2.0, shape)
    t = np.maximum(200.0, t).astype(f)
    psa = np.exp(rng.normal(0.0, 0.01, (ix, il))).astype(f)
    rh = (rng.uniform(0.3, 0.95, shape) * sig ** 2).astype(f)
    q = (rh * qsat_f32(t, psa[None], vert["fsg"][:, None, None])).astype(f)
    cos2 = np.cos(lat)[None, None, :] ** 2
    u = (25.0 * cos2 * (1.0 - sig) + rng.normal(0.0, 3.0, shape)).astype(f)
    v = rng.normal(0.0, 3.0, shape).astype(f)
    phi = (phis[None] + RGAS * t.astype(np.float64) * (-np.log(sig))).astype(f)
    return vert, t, q, u, v, psa, phi


def config0_instance(seed=0, ix=96, il=48, kx=8, lfluxland=False, tyear=80.0 / DAYS_YEAR,
                     model_step=0):
    """T31 aquaplanet column set: all ocean, SST = 271.4 + 29 cos^2(lat), no ice, day 80."""
    f = np.float32
    rng = np.random.default_rng(seed)
    lat = gaussian_latitudes(il)
    phis = np.zeros((ix, il))
    vert, t, q, u, v, psa, phi = _atmosphere(rng, kx, ix, il, lat, phis)
    sst = np.broadcast_to(271.4 + 29.0 * np.cos(lat) ** 2, (ix, il)).astype(f)
    z = np.zeros((ix, il), f)
    return Instance(kx, ix, il, u, v, t, q, phi, psa, sst.copy(), sst.copy(), z.copy(),
                    z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), z.copy(), lat,
                    np.sin(lat).astype(f), np.cos(lat).astype(f), vert, tyear=tyear,
                    model_step=model_step, lfluxland=lfluxland, name=f"T31aqua_s{seed}")


def land_instance(seed, ix, il, kx, sst_noise=0.0, tyear=80.0 / DAYS_YEAR, model_step=0):
    """Ensemble member: config-0 atmosphere over 30% land with orography, soil moisture,
    snow poleward of 50 degrees and sea ice where SST < 271.4 K."""
    from scipy.ndimage import gaussian_filter
    f = np.float32
    rng = np.random.default_rng(seed)
    lat = gaussian_latitudes(il)
    noise = gaussian_filter(rng.normal(0.0, 1.0, (ix, il)), sigma=max(1.0, ix / 32.0),
                            mode=("wrap", "nearest"))
    fmask = (noise >= np.percentile(noise, 70.0)).astype(f)
    phis = np.abs(rng.normal(0.0, 1.0, (ix, il))) * 1.5e4 * fmask
    vert, t, q, u, v, psa, phi = _atmosphere(rng, kx, ix, il, lat, phis)
    sst = 271.4 + 29.0 * np.cos(lat)[None, :] ** 2 + np.zeros((ix, il))
    if sst_noise:
        sst = sst + rng.normal(0.0, sst_noise, (ix, il))
    sice = (sst < 271.4).astype(f)
    soilw = rng.uniform(0.0, 1.0, (ix, il)).astype(f)
    depth = rng.uniform(0.0, 0.1, (ix, il)) * (np.abs(np.degrees(lat))[None, :] > 50.0) * fmask
    snowc = (depth * 1000.0 / 60.0).astype(f)
    orog = (phis / GRAV).astype(f)
    return Instance(kx, ix, il, u, v, t, q, phi, psa, sst.astype(f), sst.astype(f), soilw,
                    snowc, sice, np.full((ix, il), 0.2, f), fmask, orog,
                    (orog.astype(np.float64) * GRAV).astype(f), lat,
                    np.sin(lat).astype(f), np.cos(lat).astype(f), vert, tyear=tyear,
                    model_step=model_step, lfluxland=True, name=f"land_{ix}x{il}x{kx}_s{seed}")


ENSEMBLE_LAYOUT = ((21, 32), (31, 16), (42, 8), (85, 4), (170, 1))


def ensemble_members(base_seed=1000, layout=ENSEMBLE_LAYOUT, sst_noise=0.0, scale=1):
    """The ragged mixed-resolution ensemble, one Instance per member (seed = base + member)."""
    out, mid = [], 0
    for trunc, count in layout:
        ix, il = GRIDS[trunc]
        for n in range(max(1, count // scale) if scale > 1 else count):
            kx = 16 if (trunc == 170 or n % 2 == 1) else 8
            inst = land_instance(base_seed + mid, ix, il, kx, sst_noise=sst_noise)
            inst.name = f"T{trunc}_m{mid}_k{kx}"
            out.append(inst)
            mid += 1
    return out


def t425_instance(seed=425, kx=16):
    ix, il = GRIDS[425]
    inst = land_instance(seed, ix, il, kx)
    inst.name = "T425_k16"
    return inst


def path_bytes(kx, columns):
    """Algorithmic bytes of one forward call: u, v, T, q and phi at every level, psa, six
    forcing and three geometry fields read; four tendency planes and the two precipitation
    fields written, each once: 4 (9 kx + 12) bytes per column."""
    return 4 * (9 * kx + 12) * columns


def fwd_bytes(kx, columns):
    """Bytes a forward call must move at least: T, q, phi at every level, u and v at the lowest
    level (the only level the physics reads), psa, six forcing and three geometry fields read;
    four tendency planes and two precipitation fields written: 4 (7 kx + 14) bytes per
    column."""
    return 4 * (7 * kx + 14) * columns


def levelset_bytes(kx, columns):
    """Bytes the forward's level-set launch reads: T, q, phi at every level and psa,
    4 (3 kx + 1) per column (a re-read of the fused launch's inputs)."""
    return 4 * (3 * kx + 1) * columns
