"""The reference-facing drop-in: JAX-GCM's physics interface restated over torch CUDA tensors.

Names, fields and argument meaning follow the reference:

* ``PhysicsState`` / ``PhysicsTendency`` / ``Physics``   -- jcm/physics_interface.py:22-194
* ``ForcingData``                                         -- jcm/forcing.py:8-131
* ``DateData``                                            -- jcm/date.py:9-48
* ``Geometry``                                            -- jcm/geometry.py:62-236
* ``Parameters`` and its groups                           -- jcm/physics/speedy/params.py:9-295
* ``SpeedyPhysics.compute_tendencies``                    -- jcm/physics/speedy/speedy_physics.py:88-127
* ``get_physical_tendencies`` physics part (verify clamps) -- jcm/physics_interface.py:305-376

Fields are float32 CUDA tensors in the reference layout (``[kx, ix, il]`` level fields,
``[ix, il]`` surface fields, ``[il]`` latitude tables).  All compute goes through the C ABI of
``libspeedy_b200.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, fields, replace
from types import SimpleNamespace
from typing import Optional

import numpy as np
import torch

from . import _lib

DAYS_YEAR = 365.2425
GRAV = 9.81
P0 = 1e5
CP = 1004.0

SIGMA_LAYER_BOUNDARIES = {
    7: [0.0, 0.14, 0.26, 0.42, 0.6, 0.77, 0.9, 1.0],
    8: [0.0, 0.05, 0.14, 0.26, 0.42, 0.6, 0.77, 0.9, 1.0],
    16: [k / 16.0 for k in range(17)],
}


def _dev(x, device, dtype=torch.float32):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    a = np.asarray(x)
    if not a.flags.writeable:  # e.g. a broadcast view: torch wants its own writable copy
        a = np.array(a)
    return torch.as_tensor(a, dtype=dtype, device=device).contiguous()


# ---------------------------------------------------------------------------------------------
# State containers (physics_interface.py:22-120)
# ---------------------------------------------------------------------------------------------
@dataclass
class PhysicsState:
    u_wind: torch.Tensor
    v_wind: torch.Tensor
    temperature: torch.Tensor
    specific_humidity: torch.Tensor  # g/kg
    geopotential: torch.Tensor
    normalized_surface_pressure: torch.Tensor  # p / 1e5 Pa

    @classmethod
    def zeros(cls, shape, device="cuda", **kw):
        z = lambda s: torch.zeros(s, dtype=torch.float32, device=device)
        base = dict(u_wind=z(shape), v_wind=z(shape), temperature=z(shape),
                    specific_humidity=z(shape), geopotential=z(shape),
                    normalized_surface_pressure=z(tuple(shape[1:])))
        base.update({k: _dev(v, device) for k, v in kw.items() if v is not None})
        return cls(**base)

    @classmethod
    def ones(cls, shape, device="cuda", **kw):
        st = cls.zeros(shape, device)
        for f in fields(st):
            getattr(st, f.name).fill_(1.0)
        for k, v in kw.items():
            if v is not None:
                setattr(st, k, _dev(v, device))
        return st

    def copy(self, **kw):
        return replace(self, **{k: v for k, v in kw.items() if v is not None})


@dataclass
class PhysicsTendency:
    u_wind: torch.Tensor
    v_wind: torch.Tensor
    temperature: torch.Tensor
    specific_humidity: torch.Tensor

    @classmethod
    def zeros(cls, shape, device="cuda"):
        z = lambda: torch.zeros(shape, dtype=torch.float32, device=device)
        return cls(z(), z(), z(), z())

    def __add__(self, other):
        return PhysicsTendency(*(getattr(self, f.name) + getattr(other, f.name) for f in fields(self)))


@dataclass
class ForcingData:
    alb0: torch.Tensor
    sice_am: torch.Tensor
    snowc_am: torch.Tensor
    soilw_am: torch.Tensor
    stl_am: torch.Tensor
    sea_surface_temperature: torch.Tensor
    lfluxland: bool = False

    @classmethod
    def zeros(cls, nodal_shape, device="cuda", lfluxland=None, **kw):
        z = lambda: torch.zeros(tuple(nodal_shape), dtype=torch.float32, device=device)
        base = dict(alb0=z(), sice_am=z(), snowc_am=z(), soilw_am=z(), stl_am=z(),
                    sea_surface_temperature=z())
        base.update({k: _dev(v, device) for k, v in kw.items() if v is not None})
        return cls(**base, lfluxland=bool(lfluxland) if lfluxland is not None else False)

    @classmethod
    def ones(cls, nodal_shape, device="cuda", lfluxland=None, **kw):
        f = cls.zeros(nodal_shape, device, lfluxland=True if lfluxland is None else lfluxland)
        for n in ("alb0", "sice_am", "snowc_am", "soilw_am", "stl_am", "sea_surface_temperature"):
            getattr(f, n).fill_(1.0)
        for k, v in kw.items():
            if v is not None:
                setattr(f, k, _dev(v, device))
        return f

    def day_slice(self, day):
        """tree_index_3d(forcing, day) (jcm/utils.py:104-108): 3-D daily fields -> 2-D.  Forcing
        whose fields are all 2-D already is returned as it is."""
        names = ("alb0", "sice_am", "snowc_am", "soilw_am", "stl_am", "sea_surface_temperature")
        if all(getattr(self, n).dim() == 2 for n in names):
            return self
        out = {}
        for n in ("alb0", "sice_am", "snowc_am", "soilw_am", "stl_am", "sea_surface_temperature"):
            a = getattr(self, n)
            out[n] = a[:, :, day].contiguous() if a.dim() > 2 else a
        return ForcingData(**out, lfluxland=self.lfluxland)


@dataclass
class DateData:
    tyear: float = 0.0
    model_year: int = 1950
    model_step: int = 0
    dt_seconds: float = 1800.0

    @classmethod
    def zeros(cls, tyear=None, model_year=None, model_step=None, dt_seconds=None):
        return cls(0.0 if tyear is None else tyear, 1950 if model_year is None else model_year,
                   0 if model_step is None else model_step,
                   1800.0 if dt_seconds is None else dt_seconds)

    def model_day(self):
        """round(tyear * 365.2425) in float32, half to even (date.py:40-41)."""
        return int(np.round(np.float32(self.tyear) * np.float32(DAYS_YEAR)))


# ---------------------------------------------------------------------------------------------
# Geometry (geometry.py:62-236)
# ---------------------------------------------------------------------------------------------
def initialize_vertical(kx):
    """_initialize_vertical (geometry.py:62-85) in float32 (numpy, host side)."""
    if kx not in SIGMA_LAYER_BOUNDARIES:
        raise ValueError(f"Invalid number of vertical levels: {kx}")
    f = np.float32
    hsg = np.asarray(SIGMA_LAYER_BOUNDARIES[kx], f)
    fsg = (hsg[1:] + hsg[:-1]) / f(2.0)
    dhs = np.diff(hsg)
    sigl = np.log(fsg)
    grdsig = f(GRAV) / (dhs * f(P0))
    grdscp = grdsig / f(CP)
    wvi = np.zeros((kx, 2), f)
    wvi[:-1, 0] = f(1.0) / np.diff(sigl)
    wvi[:-1, 1] = (np.log(hsg[1:-1]) - sigl[:-1]) * wvi[:-1, 0]
    wvi[-1, 1] = (np.log(f(0.99)) - sigl[-1]) * wvi[-2, 0]
    return hsg, fsg, dhs, sigl, grdsig, grdscp, wvi


@dataclass
class Geometry:
    nodal_shape: tuple
    orog: torch.Tensor
    phis0: torch.Tensor
    fmask: torch.Tensor
    radang: np.ndarray
    sia: torch.Tensor
    coa: torch.Tensor
    hsg: np.ndarray
    fsg: np.ndarray
    dhs: np.ndarray
    sigl: np.ndarray
    grdsig: np.ndarray
    grdscp: np.ndarray
    wvi: np.ndarray
    _vgrid: Optional[object] = field(default=None, repr=False, compare=False)

    @classmethod
    def from_grid_shape(cls, nodal_shape, num_levels=8, orography=None, fmask=None, phis0=None,
                        latitudes=None, device="cuda"):
        """Geometry for an (ix, il) grid.  Latitudes default to Gauss-Legendre nodes (south to
        north); ``phis0`` defaults to ``grav * orography`` (no spectral truncation here)."""
        ix, il = nodal_shape
        if latitudes is None:
            x, _ = np.polynomial.legendre.leggauss(il)
            latitudes = np.arcsin(x)
        radang = np.asarray(latitudes, np.float64)
        orog = np.zeros((ix, il), np.float32) if orography is None else np.broadcast_to(
            np.asarray(orography, np.float32), (ix, il))
        fm = np.zeros((ix, il), np.float32) if fmask is None else np.broadcast_to(
            np.asarray(fmask, np.float32), (ix, il))
        ph = (orog.astype(np.float32) * np.float32(GRAV)) if phis0 is None else np.broadcast_to(
            np.asarray(phis0, np.float32), (ix, il))
        vert = initialize_vertical(num_levels)
        return cls((num_levels, ix, il), _dev(orog, device), _dev(ph, device), _dev(fm, device),
                   radang, _dev(np.sin(radang).astype(np.float32), device),
                   _dev(np.cos(radang).astype(np.float32), device), *vert)

    @classmethod
    def single_column_geometry(cls, radang=0.0, orog=0.0, fmask=0.0, phis0=None, num_levels=8,
                               device="cuda"):
        """geometry.py:207-236."""
        if phis0 is None:
            phis0 = GRAV * orog
        return cls.from_grid_shape((1, 1), num_levels, orography=[[orog]], fmask=[[fmask]],
                                   phis0=[[phis0]], latitudes=[radang], device=device)

    def vgrid(self):
        if self._vgrid is None:
            kx = self.nodal_shape[0]
            vg = _lib.VGrid()
            for name in ("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp"):
                arr = np.asarray(getattr(self, name), np.float32)
                tgt = getattr(vg, name)
                for i, v in enumerate(arr):
                    tgt[i] = float(v)
            for k in range(kx):
                vg.wvi[k][0] = float(self.wvi[k, 0])
                vg.wvi[k][1] = float(self.wvi[k, 1])
            self._vgrid = vg
        return self._vgrid


# ---------------------------------------------------------------------------------------------
# Parameters (params.py:9-295)
# ---------------------------------------------------------------------------------------------
@dataclass
class ConvectionParameters:
    psmin: float = 0.8
    trcnv: float = 6.0
    rhil: float = 0.7
    rhbl: float = 0.9
    entmax: float = 0.5
    smf: float = 0.8


@dataclass
class ForcingParameters:
    increase_co2: bool = False
    co2_year_ref: int = 1950


@dataclass
class CondensationParameters:
    trlsc: float = 4.0
    rhlsc: float = 0.9
    drhlsc: float = 0.1
    rhblsc: float = 0.95


@dataclass
class ShortwaveRadiationParameters:
    albcl: float = 0.43
    albcls: float = 0.50
    absdry: float = 0.033
    absaer: float = 0.033
    abswv1: float = 0.022
    abswv2: float = 15.000
    abscl1: float = 0.015
    abscl2: float = 0.15
    ablwin: float = 0.3
    ablwv1: float = 0.7
    ablwv2: float = 50.0
    ablcl1: float = 12.0
    ablcl2: float = 0.6
    rhcl1: float = 0.30
    rhcl2: float = 1.00
    qacl: float = 0.20
    wpcl: float = 0.2
    pmaxcl: float = 10.0
    clsmax: float = 0.60
    clsminl: float = 0.15
    gse_s0: float = 0.25
    gse_s1: float = 0.40


@dataclass
class ModRadConParameters:
    albsea: float = 0.07
    albice: float = 0.60
    albsn: float = 0.60
    epslw: float = 0.05
    emisfc: float = 0.98


@dataclass
class SurfaceFluxParameters:
    fwind0: float = 0.95
    ftemp0: float = 1.0
    fhum0: float = 0.0
    cdl: float = 2.4e-3
    cds: float = 1.0e-3
    chl: float = 1.2e-3
    chs: float = 0.9e-3
    vgust: float = 5.0
    ctday: float = 1.0e-2
    dtheta: float = 3.0
    fstab: float = 0.67
    clambda: float = 7.0
    clambsn: float = 7.0
    lscasym: bool = True
    lskineb: bool = True
    hdrag: float = 2000.0


@dataclass
class VerticalDiffusionParameters:
    trshc: float = 6.0
    trvdi: float = 24.0
    trvds: float = 6.0
    redshc: float = 0.5
    rhgrad: float = 0.5
    segrad: float = 0.1


GROUPS = ("convection", "condensation", "shortwave_radiation", "mod_radcon", "surface_flux",
          "vertical_diffusion", "forcing")

# The 12 scalars the adjoint differentiates (params.py:11-16, :51-54, :72-73).
DIFF_PARAMS = [("convection", "psmin"), ("convection", "trcnv"), ("convection", "rhil"),
               ("convection", "rhbl"), ("convection", "entmax"), ("convection", "smf"),
               ("condensation", "trlsc"), ("condensation", "rhlsc"),
               ("condensation", "drhlsc"), ("condensation", "rhblsc"),
               ("shortwave_radiation", "albcl"), ("shortwave_radiation", "albcls")]


@dataclass
class Parameters:
    convection: ConvectionParameters = field(default_factory=ConvectionParameters)
    condensation: CondensationParameters = field(default_factory=CondensationParameters)
    shortwave_radiation: ShortwaveRadiationParameters = field(
        default_factory=ShortwaveRadiationParameters)
    mod_radcon: ModRadConParameters = field(default_factory=ModRadConParameters)
    surface_flux: SurfaceFluxParameters = field(default_factory=SurfaceFluxParameters)
    vertical_diffusion: VerticalDiffusionParameters = field(
        default_factory=VerticalDiffusionParameters)
    forcing: ForcingParameters = field(default_factory=ForcingParameters)

    @classmethod
    def default(cls):
        return cls()

    def with_values(self, **kw):
        """Copy with ``group__name=value`` overrides."""
        groups = {g: replace(getattr(self, g)) for g in GROUPS}
        for key, val in kw.items():
            g, n = key.split("__")
            setattr(groups[g], n, val)
        return Parameters(**groups)

    def to_struct(self):
        p = _lib.Params()
        flat = {}
        for g in GROUPS[:-1]:
            for f in fields(getattr(self, g)):
                flat[f.name] = getattr(getattr(self, g), f.name)
        for name in _lib.PARAM_FIELDS:
            setattr(p, name, float(np.float32(flat[name])))
        return p

    def flags(self):
        f = 0
        if self.surface_flux.lscasym:
            f |= _lib.SPD_LSCASYM
        if self.surface_flux.lskineb:
            f |= _lib.SPD_LSKINEB
        if self.forcing.increase_co2:
            f |= _lib.SPD_INCREASE_CO2
        return f


# ---------------------------------------------------------------------------------------------
# Physics (physics_interface.py:137-194, speedy_physics.py:34-132)
# ---------------------------------------------------------------------------------------------
class Physics:
    def compute_tendencies(self, state, forcing, geometry, date):
        raise NotImplementedError("Physics compute_tendencies method not implemented.")

    def speculating(self, accumulate=False):
        """Whether a call predicts the level set (see the class docstring); accumulating
        diagnostics never does (a redone column would add its diagnostics twice)."""
        return self.speculate and not accumulate

    def get_empty_data(self, geometry):
        return None


DIAG_2D = ("cbmf", "cloudc", "cloudstr", "rsds", "rsns", "ftop_sw", "rlds", "rlns", "ftop_lw",
           "tsfc", "tskin", "shf", "evap")


def physics_data_from_diagnostics(d):
    """A PhysicsData-shaped namespace (physics_data.py:449-518) holding the kernel's diagnostic
    outputs; leaves the kernel does not produce are absent."""
    ns = SimpleNamespace
    return ns(
        convection=ns(iptop=d.get("iptop"), cbmf=d.get("cbmf"), precnv=d["precnv"]),
        condensation=ns(precls=d["precls"]),
        shortwave_rad=ns(cloudc=d.get("cloudc"), cloudstr=d.get("cloudstr"),
                         icltop=d.get("icltop"), rsds=d.get("rsds"), rsns=d.get("rsns"),
                         ftop=d.get("ftop_sw")),
        longwave_rad=ns(ftop=d.get("ftop_lw")),
        surface_flux=ns(rlds=d.get("rlds"), rlns=d.get("rlns"), tsfc=d.get("tsfc"),
                        tskin=d.get("tskin"), shf=d.get("shf"), evap=d.get("evap")),
    )


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def current_raw_stream(device_index):
    """The current CUDA stream of a device as a raw handle (torch's own fast path where it has
    one; torch.cuda.current_stream otherwise)."""
    f = getattr(torch._C, "_cuda_getCurrentRawStream", None)
    return f(device_index) if f is not None else torch.cuda.current_stream(device_index).cuda_stream


class SpeedyPhysics(Physics):
    """SPEEDY physics on the B200 (speedy_physics.py:34-132).

    ``fuse_verify=True`` also applies ``verify_state`` before and ``verify_tendencies`` after
    the physics (physics_interface.py:305-342), as ``get_physical_tendencies`` does, with
    ``time_step`` (default: ``date.dt_seconds``).  ``q_tend_scale`` multiplies the humidity
    tendency last (for the g/kg/s -> model-units conversion of
    physics_tendency_to_dynamics_tendency, physics_interface.py:286).
    ``orographic_correction=True`` appends the orographic correction as the last term
    (orographic_correction.py:177-247), which the reference's term list carries commented out
    (speedy_physics.py:65,79).

    ``speculate=True`` (the default) predicts the instance's cloud-top level set (the one
    cross-column dependency, shortwave_radiation.py:62-68) from this object's previous call
    and checks it on the device: the physics runs in one pass over the columns, and a second
    pass follows only when the prediction missed (the first call, or after another instance's
    call).  ``speculate=False`` forms the level set first in a light launch.  Both give the same
    results bitwise.  Calls of one object use one scratch buffer: order them on one stream.
    """

    def __init__(self, parameters: Optional[Parameters] = None, checkpoint_terms=True,
                 fuse_verify=False, time_step=None, q_tend_scale=1.0, diagnostics=True,
                 orographic_correction=False, speculate=True):
        self.speculate = speculate
        self.parameters = parameters or Parameters.default()
        self.fuse_verify = fuse_verify
        self.orographic_correction = orographic_correction
        self.time_step = time_step
        self.q_tend_scale = q_tend_scale
        self.diagnostics = diagnostics
        self._pstruct = self.parameters.to_struct()
        self._scratch = {}
        self._day = (None, 0)  # (tyear, model day) of the last call

    def desc(self, geometry, date, lfluxland):
        kx, ix, il = geometry.nodal_shape
        flags = self.parameters.flags()
        if lfluxland:
            flags |= _lib.SPD_LFLUXLAND
        if self.fuse_verify:
            flags |= _lib.SPD_FUSE_VERIFY
        if self.orographic_correction:
            # the term divides by the date's step (orographic_correction.py:236-238), the
            # kernel by the one step it is given
            if self.time_step is not None and float(self.time_step) != float(date.dt_seconds):
                raise ValueError("orographic_correction needs time_step == date.dt_seconds")
            flags |= _lib.SPD_OROGRAPHIC
        if not self.speculate:
            flags |= _lib.SPD_NO_SPECULATION
        dt = date.dt_seconds if self.time_step is None else self.time_step
        return _lib.Desc(kx, ix, il, flags, float(np.float32(date.tyear)), int(date.model_year),
                         int(date.model_step), int(self.parameters.forcing.co2_year_ref),
                         float(dt), float(self.q_tend_scale))

    def _scratch_for(self, desc, device):
        lib = _lib.load()
        n = lib.spd_fwd_scratch_bytes(C.byref(desc))
        key = (device, n)
        buf = self._scratch.get(key)
        if buf is None:
            buf = torch.empty(n, dtype=torch.uint8, device=device)
            self._scratch = {key: buf}
        return buf

    def compute_tendencies(self, state: PhysicsState, forcing: ForcingData, geometry: Geometry,
                           date: DateData, out: Optional[dict] = None, marker=None,
                           accumulate: bool = False):
        """Tendencies and PhysicsData for ``state``.  ``out`` may give preallocated output
        tensors (they must not overlap the inputs); ``marker`` (a torch.cuda.Event) is recorded
        between the call's two launches, for timing them separately: after the fused launch
        (before the fixup) when speculating, after the level-set launch (before the fused one)
        otherwise (``speculating(accumulate)`` says which).  ``accumulate=True`` adds precnv, precls and the float
        diagnostics to what ``out`` holds instead of overwriting them (the running sums of
        DiagnosticsCollector, jcm/model.py:46-64; scale by 1/steps once at the end)."""
        if accumulate and out is None:
            raise ValueError("accumulate=True adds into `out`: pass the running sums")
        lib = _lib.load()
        kx, ix, il = geometry.nodal_shape
        t = state.temperature
        if tuple(t.shape) != (kx, ix, il):
            raise ValueError(f"state shape {tuple(t.shape)} does not match geometry {(kx, ix, il)}")
        if not t.is_cuda:
            raise RuntimeError("SpeedyPhysics runs on CUDA tensors only (no CPU path)")
        dev = t.device
        didx = t.get_device()
        _lib.preload(didx)
        if self._day[0] != date.tyear:
            self._day = (date.tyear, date.model_day())
        f2 = forcing.day_slice(self._day[1])
        tensors = dict(u_wind=state.u_wind, v_wind=state.v_wind, temperature=state.temperature,
                       specific_humidity=state.specific_humidity,
                       geopotential=state.geopotential,
                       normalized_surface_pressure=state.normalized_surface_pressure,
                       alb0=f2.alb0, sice_am=f2.sice_am, snowc_am=f2.snowc_am,
                       soilw_am=f2.soilw_am, stl_am=f2.stl_am,
                       sea_surface_temperature=f2.sea_surface_temperature, fmask=geometry.fmask,
                       orog=geometry.orog, phis0=geometry.phis0, sia=geometry.sia,
                       coa=geometry.coa)
        ptrs = []
        for k in _lib.INPUT_FIELDS:
            v = tensors[k]
            if v.dtype is not torch.float32 or not v.is_contiguous() or v.get_device() != didx:
                v = tensors[k] = v.to(device=dev, dtype=torch.float32).contiguous()
            ptrs.append(v.data_ptr())
        if out is None:
            e3 = lambda: torch.empty((kx, ix, il), dtype=torch.float32, device=dev)
            e2 = lambda: torch.empty((ix, il), dtype=torch.float32, device=dev)
            out = dict(u_wind=e3(), v_wind=e3(), temperature=e3(), specific_humidity=e3(),
                       precnv=e2(), precls=e2())
            if self.diagnostics:
                for n in DIAG_2D:
                    out[n] = e2()
                out["iptop"] = torch.empty((ix, il), dtype=torch.int32, device=dev)
                out["icltop"] = torch.empty((ix, il), dtype=torch.int32, device=dev)
        inp = _lib.Inputs(*ptrs)
        outs = _lib.Outputs(*[out[k].data_ptr() if k in out else None
                              for k in _lib.OUTPUT_FIELDS])
        desc = self.desc(geometry, date, forcing.lfluxland)
        if accumulate:
            desc.flags |= _lib.SPD_ACCUMULATE_DIAGNOSTICS
        scratch = self._scratch_for(desc, dev)
        stream = current_raw_stream(didx)
        ev = C.c_void_p(marker.cuda_event) if marker is not None else None
        rc = lib.spd_fwd_marked(C.byref(desc), C.byref(geometry.vgrid()), C.byref(self._pstruct),
                                C.byref(inp), C.byref(outs), _ptr(scratch), scratch.numel(),
                                C.c_void_p(stream), ev)
        _lib.check(rc, "spd_fwd")
        tend = PhysicsTendency(out["u_wind"], out["v_wind"], out["temperature"],
                               out["specific_humidity"])
        return tend, physics_data_from_diagnostics(out)

    def get_empty_data(self, geometry):
        return None


def get_physical_tendencies_columns(state, physics, forcing, geometry, date, time_step):
    """The column part of get_physical_tendencies (physics_interface.py:371-376): verify_state,
    compute_tendencies and verify_tendencies fused into the kernel.  The spectral transforms
    around it (dinosaur) stay with the caller."""
    phys = physics if physics.fuse_verify else SpeedyPhysics(
        physics.parameters, fuse_verify=True, time_step=time_step,
        q_tend_scale=physics.q_tend_scale, diagnostics=physics.diagnostics,
        orographic_correction=physics.orographic_correction)
    phys.time_step = time_step
    return phys.compute_tendencies(state, forcing, geometry, date)


def instance_to_device(inst, device="cuda"):
    """(PhysicsState, ForcingData, Geometry, DateData) on ``device`` for a synthetic Instance
    (``synthetic.py``)."""
    dev = torch.device(device)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32, device=dev)
    state = PhysicsState(t(inst.u), t(inst.v), t(inst.t), t(inst.q), t(inst.phi), t(inst.psa))
    forcing = ForcingData(t(inst.alb0), t(inst.sice), t(inst.snowc), t(inst.soilw),
                          t(inst.stl), t(inst.sst), lfluxland=inst.lfluxland)
    geom = Geometry.from_grid_shape((inst.ix, inst.il), inst.kx, orography=inst.orog,
                                    fmask=inst.fmask, phis0=inst.phis0, latitudes=inst.lat,
                                    device=dev)
    geom.sia, geom.coa = t(inst.sia), t(inst.coa)
    date = DateData(inst.tyear, inst.model_year, inst.model_step, inst.dt_seconds)
    return state, forcing, geom, date
