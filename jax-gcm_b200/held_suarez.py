"""Held-Suarez physics on the B200: the drop-in for ``HeldSuarezPhysics``
(jcm/physics/held_suarez/held_suarez_physics.py:14-101), the reference's second physics
package, through ``spd_held_suarez``.

The constructor takes the reference's coefficients.  The reference nondimensionalizes them with
dinosaur's scales; here they are plain numbers in the caller's units (the defaults are SI: rates
in 1/s, temperatures in K, giving tendencies in K/s and m/s^2), and the arithmetic is the same.
Level centres and latitudes come from the Geometry (``fsg``, ``radang``), as the reference takes
them from its coordinate system.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np
import torch

from . import _lib
from .physics import Geometry, Physics, PhysicsState, PhysicsTendency

DAY = 86400.0


class HeldSuarezPhysics(Physics):
    def __init__(self, sigma_b: float = 0.7, kf: float = 1.0 / DAY, ka: float = 1.0 / (40 * DAY),
                 ks: float = 1.0 / (4 * DAY), minT: float = 200.0, maxT: float = 315.0,
                 dTy: float = 60.0, dThz: float = 10.0, kappa: float = 2.0 / 7.0):
        self.sigma_b, self.kf, self.ka, self.ks = sigma_b, kf, ka, ks
        self.minT, self.maxT, self.dTy, self.dThz, self.kappa = minT, maxT, dTy, dThz, kappa
        self._tables = {}

    def _desc(self, geometry: Geometry):
        kx, ix, il = geometry.nodal_shape
        d = _lib.HsDesc()
        d.kx, d.ix, d.il = kx, ix, il
        d.sigma_b, d.kf, d.ka, d.ks = self.sigma_b, self.kf, self.ka, self.ks
        d.min_t, d.max_t, d.dt_y, d.dthz, d.kappa = (self.minT, self.maxT, self.dTy, self.dThz,
                                                     self.kappa)
        for k in range(kx):
            d.sigma[k] = float(np.float32(geometry.fsg[k]))
        return d

    def _lat_table(self, geometry: Geometry, device):
        """sin^2, cos^2, cos^4 of the latitudes, formed in float32 as the reference does
        (held_suarez_physics.py:58-61, :72-73), on the device (cached per geometry)."""
        key = (id(geometry), str(device))
        tab = self._tables.get(key)
        if tab is None:
            la = np.asarray(geometry.radang, np.float64).astype(np.float32)
            host = np.stack([np.sin(la) ** 2, np.cos(la) ** 2, np.cos(la) ** 4]).astype(np.float32)
            tab = torch.as_tensor(host, device=device).contiguous()
            self._tables = {key: tab}
        return tab

    def compute_tendencies(self, state: PhysicsState, forcing=None,
                           geometry: Optional[Geometry] = None, date=None, out=None):
        """Tendencies of ``state`` (u, v, T, normalized surface pressure on the CUDA device);
        returns (PhysicsTendency, None) like the reference.  ``out`` may give preallocated
        u_wind, v_wind, temperature, specific_humidity tensors."""
        if geometry is None:
            raise ValueError("HeldSuarezPhysics needs the Geometry (level centres, latitudes)")
        lib = _lib.load()
        t = state.temperature
        if t.device.type != "cuda":
            raise RuntimeError("HeldSuarezPhysics runs on CUDA tensors only (no CPU path)")
        if tuple(t.shape) != tuple(geometry.nodal_shape):
            raise ValueError(f"state shape {tuple(t.shape)} does not match geometry "
                             f"{tuple(geometry.nodal_shape)}")
        dev = t.device
        _lib.preload(dev.index if dev.index is not None else torch.cuda.current_device())
        f = lambda x: x.to(device=dev, dtype=torch.float32).contiguous()
        u, v, tt, ps = (f(state.u_wind), f(state.v_wind), f(t),
                        f(state.normalized_surface_pressure))
        if out is None:
            out = {k: torch.empty_like(tt) for k in ("u_wind", "v_wind", "temperature",
                                                      "specific_humidity")}
        tab = self._lat_table(geometry, dev)
        p = lambda x: C.c_void_p(x.data_ptr())
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.spd_held_suarez(C.byref(self._desc(geometry)), p(tab), p(u), p(v), p(tt), p(ps),
                                 p(out["u_wind"]), p(out["v_wind"]), p(out["temperature"]),
                                 p(out["specific_humidity"]), C.c_void_p(stream))
        _lib.check(rc, "spd_held_suarez")
        return PhysicsTendency(out["u_wind"], out["v_wind"], out["temperature"],
                               out["specific_humidity"]), None
