"""Oracle: a NumPy restatement of JAX-GCM's Held-Suarez physics.

TEST INFRASTRUCTURE ONLY.  The parity checker for ``spd_held_suarez``; only ``tests/`` and
``bench.py``'s CPU baseline leg may import it.  Each function restates one method of
``HeldSuarezPhysics`` (jcm/physics/held_suarez/held_suarez_physics.py) in ``dtype`` (float32,
the parity target, or float64 for the x64 report).  The reference's own tests
(held_suarez_test.py) only check that a Model run stays finite, so beyond this restatement the
path's parity is pinned by the properties the reference's equations imply (tests in
tests/test_held_suarez.py).
"""
from __future__ import annotations

import numpy as np

DAY = 86400.0
KAPPA = 2.0 / 7.0  # dinosaur PHYSICS_SPECS.kappa = R / cp


def default_coefficients():
    """The constructor defaults (held_suarez_physics.py:15-25) in SI units."""
    return dict(sigma_b=0.7, kf=1.0 / DAY, ka=1.0 / (40.0 * DAY), ks=1.0 / (4.0 * DAY),
                min_t=200.0, max_t=315.0, dt_y=60.0, dthz=10.0)


def latitude_tables(lat, dtype=np.float32):
    """sin(lat)^2, cos(lat)^2, cos(lat)^4 as the reference forms them (float32 lat)."""
    la = np.asarray(lat).astype(dtype)
    return np.sin(la) ** 2, np.cos(la) ** 2, np.cos(la) ** 4


def equilibrium_temperature(sigma, psa, s2, c2, co, dtype=np.float32):
    """equilibrium_temperature (held_suarez_physics.py:53-62)."""
    p = sigma.astype(dtype)[:, None, None] * psa.astype(dtype)
    with np.errstate(all="ignore"):
        t = p ** dtype(KAPPA) * (dtype(co["max_t"]) - dtype(co["dt_y"]) * s2
                                 - dtype(co["dthz"]) * np.log(p) * c2)
    return np.maximum(dtype(co["min_t"]), t).astype(dtype)


def cutoff(sigma, co, dtype=np.float32):
    """max(0, (sigma - sigma_b) / (1 - sigma_b)) (held_suarez_physics.py:65-67, :71)."""
    sb = dtype(co["sigma_b"])
    return np.maximum(dtype(0), (sigma.astype(dtype) - sb) / (dtype(1) - sb))


def compute_tendencies(u, v, t, psa, sigma, lat, co=None, dtype=np.float32):
    """HeldSuarezPhysics.compute_tendencies (held_suarez_physics.py:76-101): (du, dv, dT, dq)."""
    co = co or default_coefficients()
    s2, c2, c4 = latitude_tables(lat, dtype)
    s2, c2, c4 = s2[None, None, :], c2[None, None, :], c4[None, None, :]
    teq = equilibrium_temperature(sigma, psa, s2, c2, co, dtype)
    cut = cutoff(sigma, co, dtype)[:, None, None]
    kv = dtype(co["kf"]) * cut
    ka, ks = dtype(co["ka"]), dtype(co["ks"])
    kt = ka + (ks - ka) * (cut * c4)
    d_t = -kt * (t.astype(dtype) - teq)
    d_v = -kv * v.astype(dtype)
    d_u = -kv * u.astype(dtype)
    d_q = np.zeros_like(t, dtype=dtype)
    return d_u.astype(dtype), d_v.astype(dtype), d_t.astype(dtype), d_q
