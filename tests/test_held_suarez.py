"""Held-Suarez forcing (jcm/physics/held_suarez/held_suarez_physics.py) through
``spd_held_suarez``: the oracle restatement's properties (CPU) and the CUDA path against it
(GPU).  The reference's own tests only run a Model and check for NaNs, so the oracle is pinned
by the equations' properties: the equilibrium temperature's bounds and its closed form at the
surface, no drag above sigma_b, relaxation towards it at the rates ka..ks."""
import importlib

import numpy as np
import pytest

from oracle import held_suarez_oracle as H

pkg = importlib.import_module("jax-gcm_b200")


def _state(seed, kx, ix, il):
    inst = pkg.synthetic.land_instance(seed, ix, il, kx)
    return inst


def test_oracle_properties():
    kx, ix, il = 16, 32, 16
    inst = _state(3, kx, ix, il)
    _, fsg, *_ = __import__("oracle.speedy_oracle", fromlist=["x"]).vertical_tables(kx)
    co = H.default_coefficients()
    du, dv, dt, dq = H.compute_tendencies(inst.u, inst.v, inst.t, inst.psa, fsg, inst.lat, co)
    s2, c2, c4 = H.latitude_tables(inst.lat)
    teq = H.equilibrium_temperature(fsg, inst.psa, s2[None, None], c2[None, None], co)
    assert teq.min() >= co["min_t"] and teq.max() <= co["max_t"] * 1.01
    # at p = p0 the equilibrium temperature is maxT - dTy sin^2(lat) (the log term vanishes)
    one = H.equilibrium_temperature(np.ones(1, np.float32), np.ones((ix, il), np.float32),
                                    s2[None, None], c2[None, None], co)
    np.testing.assert_allclose(one[0], np.broadcast_to(315.0 - 60.0 * s2, (ix, il)), rtol=1e-6)
    above = fsg <= co["sigma_b"]
    assert np.all(du[above] == 0) and np.all(dv[above] == 0) and np.all(dq == 0)
    rate = -dt / (inst.t - teq)
    assert np.all(rate[np.abs(inst.t - teq) > 1] >= co["ka"] * 0.999)
    assert np.all(rate[np.abs(inst.t - teq) > 1] <= co["ks"] * 1.001)


def test_library_rejects_overlapping_outputs():
    L = pkg._lib
    lib = L.load()
    d = L.HsDesc()
    d.kx, d.ix, d.il = 8, 4, 4
    base = 1 << 36
    ptr = lambda i: base + i * (1 << 20)
    # du on top of u: rejected before any device work
    rc = lib.spd_held_suarez(d, ptr(9), ptr(0), ptr(1), ptr(2), ptr(3), ptr(0), ptr(5), ptr(6),
                             ptr(7), None)
    assert rc == 9


@pytest.mark.gpu
@pytest.mark.parametrize("kx,ix,il", [(8, 96, 48), (16, 128, 64), (16, 7, 5), (7, 64, 32)])
def test_gpu_matches_oracle(kx, ix, il):
    import torch
    inst = _state(40 + kx + ix, kx, ix, il)
    st, fo, ge, da = pkg.instance_to_device(inst, "cuda")
    phys = pkg.HeldSuarezPhysics()
    tend, none = phys.compute_tendencies(st, fo, ge, da)
    assert none is None
    torch.cuda.synchronize()
    got = [x.cpu().numpy() for x in (tend.u_wind, tend.v_wind, tend.temperature,
                                     tend.specific_humidity)]
    ref32 = H.compute_tendencies(inst.u, inst.v, inst.t, inst.psa, ge.fsg, inst.lat)
    ref64 = H.compute_tendencies(inst.u, inst.v, inst.t, inst.psa, ge.fsg, inst.lat,
                                 dtype=np.float64)
    for name, g, r, r64 in zip(("u", "v", "t", "q"), got, ref32, ref64):
        scale = max(float(np.max(np.abs(r))), 1e-30)
        err = float(np.max(np.abs(g - r))) / scale
        err64 = float(np.max(np.abs(g - r64))) / scale
        own64 = float(np.max(np.abs(r - r64))) / scale
        print(name, f"{err:.1e}", f"{err64:.1e}", f"{own64:.1e}")
        assert err <= 1e-5, (name, err)
        assert err64 <= max(1e-5, 3 * own64), (name, err64, own64)
