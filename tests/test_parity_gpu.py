"""Parity of the CUDA path (through the C ABI) with the NumPy oracle on seeded inputs.

Bar (tests/helpers.py), per tendency and precipitation field f, element by element:
|cuda - oracle32| <= 1e-5 max(|oracle32|, floor_f max|oracle32_f|), with the per-field floors
of helpers.ELEM_FLOOR; normwise |cuda - oracle32| <= 1e-5 max|oracle32_f| as well.  For the
diagnostic fields (cloud cover, surface radiation) the normwise bar is max(1e-5, 2x the float32
oracle's own normwise error against the float64 oracle on the same inputs).  Integer levels
(iptop, icltop) exact.  Columns outside the bar must have a threshold test within 64 float32
ulps in the oracle (a trigger flip); they are counted (within 1, 4 and 64 ulps) and bounded.
Over the other columns the CUDA path's normwise error against float64 must be within
max(1e-5, 3x the float32 oracle's own).
"""
import importlib

import numpy as np
import pytest

from tests.helpers import parity_check

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


def check(pkg, inst, params=None, max_flip_frac=2e-3, **kw):
    return parity_check(pkg, inst, params=params, max_flip_frac=max_flip_frac, **kw)


@pytest.mark.parametrize("lfluxland", [False, True])
@pytest.mark.parametrize("model_step", [0, 1])
def test_t31_aquaplanet(pkg, lfluxland, model_step):
    inst = pkg.synthetic.config0_instance(seed=11, lfluxland=lfluxland, model_step=model_step)
    check(pkg, inst)


@pytest.mark.parametrize("kx", [8, 16])
def test_land_member(pkg, kx):
    inst = pkg.synthetic.land_instance(101 + kx, 64, 32, kx)
    check(pkg, inst)


def test_large_member_flip_statistics(pkg):
    """T85 with 16 levels (32,768 columns, land, orography, sea ice): the more columns, the
    likelier a convection or condensation trigger within a few float32 ulps of its threshold;
    every column outside the bar must be such a flip (explained by the oracle's recorded
    margins), and at most 0.2 % of the columns may flip (measured: none)."""
    inst = pkg.synthetic.land_instance(85, 256, 128, 16, sst_noise=1.5)
    _, summ = check(pkg, inst)
    assert summ["columns"] == 256 * 128


def test_land_member_with_sea_ice(pkg):
    inst = pkg.synthetic.land_instance(5, 128, 64, 8, sst_noise=1.5)
    assert inst.sice.sum() > 0
    check(pkg, inst)


def test_seven_levels(pkg):
    inst = pkg.synthetic.land_instance(77, 64, 32, 7)
    check(pkg, inst)


@pytest.mark.parametrize("kx", [8, 16])
def test_orographic_correction(pkg, kx):
    """The optional last term (orographic_correction.py:177-247) on a land member with
    orography, against the oracle with the same term."""
    inst = pkg.synthetic.land_instance(61 + kx, 96, 48, kx)
    assert inst.phis0.max() > 0
    check(pkg, inst, orographic_correction=True)


def test_orographic_correction_fused_verify(pkg):
    inst = pkg.synthetic.land_instance(63, 64, 32, 8)
    rng = np.random.default_rng(3)
    mask = rng.uniform(size=inst.q.shape) < 0.05
    inst.q = np.where(mask, -np.abs(inst.q) * 0.01 - 1e-4, inst.q).astype(np.float32)
    check(pkg, inst, fuse_verify=True, orographic_correction=True, time_step=1800.0)


def test_fused_verify_with_negative_humidity(pkg):
    inst = pkg.synthetic.land_instance(9, 64, 32, 8)
    rng = np.random.default_rng(0)
    mask = rng.uniform(size=inst.q.shape) < 0.05
    inst.q = np.where(mask, -np.abs(inst.q) * 0.01 - 1e-4, inst.q).astype(np.float32)
    check(pkg, inst, fuse_verify=True)


def test_single_column(pkg):
    inst = pkg.synthetic.land_instance(3, 1, 1, 8)
    check(pkg, inst)


def test_cloud_top_level_set_crosses_columns(pkg):
    """One column's cloud-top level changes another column's result, as in the reference."""
    inst = pkg.synthetic.config0_instance(seed=2, ix=4, il=2, lfluxland=True)
    check(pkg, inst)
    inst2 = pkg.synthetic.config0_instance(seed=2, ix=4, il=2, lfluxland=True)
    # saturate column (0,0) near level 2 so its icltop moves; others keep their inputs
    inst2.q[2, 0, 0] = inst2.q[2, 0, 0] * 40.0
    check(pkg, inst2)


def test_diagnostics_and_levels(pkg):
    inst = pkg.synthetic.land_instance(21, 96, 48, 8)
    rep, _ = check(pkg, inst)
    assert rep["icltop"]["nbad"] == 0 and rep["iptop"]["nbad"] == 0


def test_accumulated_diagnostics_equal_the_sum_of_calls(pkg):
    """SPD_ACCUMULATE_DIAGNOSTICS: two accumulating calls (shortwave on, then off) into zeroed
    buffers give exactly the sum of the two plain calls' diagnostics; the tendencies are the
    second call's own."""
    import dataclasses
    import torch
    inst = pkg.synthetic.land_instance(71, 64, 32, 16)
    st, fo, ge, da = pkg.instance_to_device(inst, "cuda")
    phys = pkg.SpeedyPhysics()
    dates = [da, dataclasses.replace(da, model_step=int(da.model_step) + 1)]
    plain = []
    for d in dates:
        tend, data = phys.compute_tendencies(st, fo, ge, d)
        plain.append((tend, data))
    kx, ix, il = inst.kx, inst.ix, inst.il
    e3 = lambda: torch.empty((kx, ix, il), dtype=torch.float32, device="cuda")
    out = dict(u_wind=e3(), v_wind=e3(), temperature=e3(), specific_humidity=e3())
    diag = ("precnv", "precls") + pkg.physics.DIAG_2D
    for n in diag:
        out[n] = torch.zeros((ix, il), dtype=torch.float32, device="cuda")
    for n in ("iptop", "icltop"):
        out[n] = torch.empty((ix, il), dtype=torch.int32, device="cuda")
    for d in dates:
        tend, _ = phys.compute_tendencies(st, fo, ge, d, out=out, accumulate=True)
    torch.cuda.synchronize()
    assert torch.equal(tend.temperature, plain[1][0].temperature)
    flat = lambda data: {"precnv": data.convection.precnv, "precls": data.condensation.precls,
                         "rsds": data.shortwave_rad.rsds, "cloudc": data.shortwave_rad.cloudc,
                         "rlds": data.surface_flux.rlds, "evap": data.surface_flux.evap,
                         "ftop_lw": data.longwave_rad.ftop}
    a, b = flat(plain[0][1]), flat(plain[1][1])
    for k in a:
        assert torch.equal(out[k], a[k] + b[k]), k
    with pytest.raises(ValueError):
        phys.compute_tendencies(st, fo, ge, da, accumulate=True)


@pytest.mark.parametrize("switch", ["lscasym_off", "lskineb_off", "increase_co2",
                                    "q_tend_scale_fused_verify"])
def test_reference_switches(pkg, switch):
    """The reference's non-default switches on a land member with sea ice: symmetric stability
    correction (params.py:180), no skin-temperature energy balance (params.py:181), CO2
    absorptivity growing with the model year (params.py:34, forcing.py:37-39), and the humidity
    tendency's unit scale applied after verify_tendencies (physics_interface.py:286)."""
    inst = pkg.synthetic.land_instance(131, 96, 48, 8, sst_noise=1.5)
    params, kw = None, {}
    if switch == "lscasym_off":
        params = {"surface_flux.lscasym": False}
    elif switch == "lskineb_off":
        params = {"surface_flux.lskineb": False}
    elif switch == "increase_co2":
        params = {"forcing.increase_co2": True}
        inst.model_year = 2010  # ablco2 = 6 exp(0.005 (2010 + tyear - 1950))
    else:
        rng = np.random.default_rng(4)
        mask = rng.uniform(size=inst.q.shape) < 0.05
        inst.q = np.where(mask, -np.abs(inst.q) * 0.01 - 1e-4, inst.q).astype(np.float32)
        kw = dict(fuse_verify=True, time_step=1800.0, q_tend_scale=1e-3)  # g/kg/s -> kg/kg/s
    check(pkg, inst, params=params, **kw)


def test_t425_single_instance(pkg):
    """The large single instance the T425 benchmark times: 1280x640 = 819,200 columns at 16
    levels with land, orography, snow and sea ice, the same seed as the benchmark."""
    inst = pkg.synthetic.t425_instance()
    _, summ = check(pkg, inst)
    assert summ["columns"] == 1280 * 640
