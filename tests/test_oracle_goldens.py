"""Pins the NumPy oracle against the reference's own golden vectors and known-answer tests.

Each test restates one test of ``jcm/physics/speedy/*_test.py`` (same inputs, same
tolerances); the expected values come from ``tests/golden/reference_goldens.npz``, which
``tests/golden/make_golden.py`` extracts from the reference sources.
"""
import numpy as np
import pytest

from oracle import speedy_oracle as O

F32 = np.float32
IX, IL, KX = 96, 48, 8
XY, ZXY = (IX, IL), (KX, IX, IL)


def g(goldens, key):
    return goldens[key]


@pytest.fixture(scope="module")
def params():
    return O.default_parameters()


@pytest.fixture(scope="module")
def geom():
    return O.make_geometry(IX, IL, KX, lat="speedy")


def _data(**kw):
    d = O.zeros_data(XY, KX, O.make_date())
    for path, val in kw.items():
        grp, name = path.split("__")
        setattr(getattr(d, grp), name, val)
    return d


def _varying(geom):
    fsg = geom.fsg
    ta = F32(300) * np.ones(ZXY, F32) * (fsg[:, None, None] ** (
        F32(0.05) * np.cos(F32(3) * np.arange(IL, dtype=F32) / F32(IL)) ** 3))
    ps = np.ones(XY, F32)
    qsat = O.get_qsat(ta, ps, fsg[:, None, None])
    qa = np.sin(F32(2) * np.arange(IX, dtype=F32)[:, None] / F32(IX)) ** 2 * qsat * F32(3.5)
    phi = F32(O.RGAS) * ta * np.log(fsg[:, None, None])
    return ta.astype(F32), ps, qsat.astype(F32), qa.astype(F32), phi.astype(F32)


# ---- convection_test.py -------------------------------------------------------------------
def test_diagnose_convection_varying(goldens, params, geom):
    ta, ps, qsat, qa, phi = _varying(geom)
    se = F32(O.CP) * ta + phi
    iptop, qdif = O.diagnose_convection(ps, se, qa, qsat, params, None, geom)
    np.testing.assert_allclose(iptop, goldens["npy::iptop"], atol=1e-4)
    np.testing.assert_allclose(qdif, goldens["npy::qdif"], atol=1e-4)


def test_diagnose_convection_isothermal(goldens, params, geom):
    se = g(goldens, "convection_test::test_diagnose_convection_isothermal::0").astype(F32)
    qa = g(goldens, "convection_test::test_diagnose_convection_isothermal::1").astype(F32)
    qsat = O.get_qsat(np.ones((1, 1, 1), F32) * F32(288), np.ones((1, 1, 1), F32),
                      geom.fsg[:, None, None])
    b = lambda a: np.tile(np.asarray(a, F32).reshape(KX, 1, 1), (1, IX, IL))
    itop, qdif = O.diagnose_convection(np.ones(XY, F32), b(se), b(qa), b(qsat), params, None, geom)
    assert np.all(itop == 9) and np.allclose(qdif, 0)


def test_diagnose_convection_moist_adiabat(goldens, params, geom):
    key = "convection_test::test_diagnose_convection_moist_adiabat::"
    se, qa, qsat = (goldens[key + str(i)].astype(F32) for i in range(3))
    b = lambda a: np.tile(a.reshape(KX, 1, 1), (1, IX, IL))
    itop, qdif = O.diagnose_convection(np.ones(XY, F32), b(se), b(qa) * F32(1000),
                                       b(qsat) * F32(1000), params, None, geom)
    assert itop[0, 0] == goldens[key + "assign::test_itop"]
    assert abs(qdif[0, 0] - goldens[key + "assign::test_qdif"]) < 0.5e-4


def test_convection_tendencies_varying(goldens, params, geom):
    ta, ps, qsat, qa, phi = _varying(geom)
    state = O.make_state(ZXY, temperature=ta, geopotential=phi, specific_humidity=qa,
                         normalized_surface_pressure=ps)
    data = _data(humidity__qsat=qsat)
    tend, data = O.get_convection_tendencies(state, data, params, None, geom)
    np.testing.assert_allclose(data.convection.iptop, goldens["npy::iptop"], atol=1e-4)
    np.testing.assert_allclose(data.convection.cbmf, goldens["npy::cbmf"], atol=1e-4)
    np.testing.assert_allclose(data.convection.precnv, goldens["npy::precnv"], atol=1e-4)
    dfse, dfqa = goldens["npy::dfse"], goldens["npy::dfqa"]
    tt = dfse.copy()
    tt[1:] = dfse[1:] * (1 / ps) * geom.grdscp[1:, None, None]
    qt = dfqa.copy()
    qt[1:] = dfqa[1:] * (1 / ps) * geom.grdsig[1:, None, None]
    np.testing.assert_allclose(tend.temperature, tt, atol=1e-4)
    np.testing.assert_allclose(tend.specific_humidity, qt, atol=1e-4)


def test_convection_tendencies_isothermal(goldens, params, geom):
    se = goldens["convection_test::test_get_convection_tendencies_isothermal::0"].astype(F32) / F32(O.CP)
    qa = goldens["convection_test::test_get_convection_tendencies_isothermal::1"].astype(F32)
    qsat = O.get_qsat(np.ones((1, 1, 1), F32) * F32(288), np.ones((1, 1, 1), F32),
                      geom.fsg[:, None, None])
    b = lambda a: np.tile(np.asarray(a, F32).reshape(KX, 1, 1), (1, IX, IL))
    state = O.make_state(ZXY, temperature=b(se), geopotential=np.zeros(ZXY, F32),
                         specific_humidity=b(qa), normalized_surface_pressure=np.ones(XY, F32))
    tend, data = O.get_convection_tendencies(state, _data(humidity__qsat=b(qsat)), params, None, geom)
    assert np.all(data.convection.iptop == 9)
    assert np.allclose(data.convection.cbmf, 0) and np.allclose(data.convection.precnv, 0)
    assert np.allclose(tend.temperature, 0) and np.allclose(tend.specific_humidity, 0)


def test_convection_tendencies_moist_adiabat(goldens, params, geom):
    key = "convection_test::test_get_convection_tendencies_moist_adiabat::"
    se = goldens[key + "0"].astype(F32) / F32(O.CP)
    qa, qsat = goldens[key + "1"].astype(F32), goldens[key + "2"].astype(F32)
    dfse, dfqa = goldens[key + "3"], goldens[key + "4"]
    b = lambda a: np.tile(a.reshape(KX, 1, 1), (1, IX, IL))
    state = O.make_state(ZXY, temperature=b(se), geopotential=np.zeros(ZXY, F32),
                         specific_humidity=b(qa) * F32(1000),
                         normalized_surface_pressure=np.ones(XY, F32))
    tend, data = O.get_convection_tendencies(state, _data(humidity__qsat=b(qsat) * F32(1000)),
                                             params, None, geom)
    assert abs(data.convection.cbmf[0, 0] - goldens[key + "assign::test_cbmf"]) < 0.5e-4
    assert abs(data.convection.precnv[0, 0] - goldens[key + "assign::test_precnv"]) < 0.5e-4
    tt = dfse.copy()
    tt[1:] = dfse[1:] * geom.grdscp[1:]
    qt = dfqa.copy()
    qt[1:] = dfqa[1:] * geom.grdsig[1:]
    for k in (4, 5, 6):
        assert abs(tend.temperature[k, 0, 0] - tt[k]) < 0.5e-2
        assert abs(tend.specific_humidity[k, 0, 0] - qt[k]) < 0.5e-2


# ---- large_scale_condensation_test.py -----------------------------------------------------
def test_lsc_realistic(goldens, params):
    key = "large_scale_condensation_test::test_get_large_scale_condensation_tendencies_realistic::"
    geom1 = O.make_geometry(1, 1, KX, lat=[0.0])
    xy, zxy = (1, 1), (KX, 1, 1)
    psa = F32(1.0110737) * np.ones(xy, F32)
    qa = goldens[key + "0"].astype(F32)[:, None, None] * np.ones(zxy, F32)
    qsat = goldens[key + "1"].astype(F32)[:, None, None] * np.ones(zxy, F32)
    data = O.zeros_data(xy, KX, O.make_date())
    data.humidity.qsat = qsat
    data.convection.iptop = np.ones(xy, np.int64) * 4
    state = O.make_state(zxy, specific_humidity=qa, normalized_surface_pressure=psa)
    tend, data = O.get_large_scale_condensation_tendencies(state, data, params, None, geom1)
    np.testing.assert_allclose(tend.temperature[:, 0, 0], goldens[key + "2"], atol=1e-4, rtol=0)
    np.testing.assert_allclose(tend.specific_humidity[:, 0, 0], goldens[key + "3"], atol=1e-4, rtol=0)
    assert abs(data.condensation.precls[0, 0] - goldens[key + "4"][0]) <= 0.05
    assert data.convection.iptop[0, 0] == goldens[key + "5"][0, 0]


# ---- shortwave_radiation_test.py ----------------------------------------------------------
def test_solar(goldens, geom):
    key = "shortwave_radiation_test::test_solar::"
    for n, ty in enumerate([0.2, 0.4, 0.6, 0.8, 1.0]):
        assert np.allclose(O.solar(ty, geometry=geom), goldens[key + str(n)], atol=1e-4), ty
    assert np.allclose(O.solar(0.6, 1300, geometry=geom), goldens[key + "5"], atol=1e-4)


def _sw_case(goldens, params):
    key = "shortwave_radiation_test::test_shortwave_radiation::"
    qa = F32(0.5) * F32(1000.0) * goldens[key + "0"].astype(F32)
    qsat = F32(1000.0) * goldens[key + "1"].astype(F32)
    with np.errstate(all="ignore"):
        rh = qa / qsat
    geop = np.arange(7, -1, -1).astype(F32)
    se = F32(0.1) * geop
    b = lambda a: np.tile(a[:, None, None], (1,) + XY)
    qa, qsat, rh, geop, se = b(qa), b(qsat), b(rh), b(geop), b(se)
    geom = O.make_geometry(IX, IL, KX, lat="speedy", fmask=0.7)
    data = O.zeros_data(XY, KX, O.make_date(tyear=0.6))
    data.humidity.rh, data.humidity.qsat = rh, qsat
    data.convection.iptop = 8 * np.ones(XY, np.int64)
    data.convection.precnv = -1.0 * np.ones(XY, F32)
    data.convection.se = se
    data.condensation.precls = 4.0 * np.ones(XY, F32)
    data.shortwave_rad.compute_shortwave = True
    state = O.make_state(ZXY, specific_humidity=qa, geopotential=geop,
                         normalized_surface_pressure=np.ones(XY, F32))
    forcing = O.make_forcing(XY)
    _, data = O.get_clouds(state, data, params, forcing, geom)
    data = O.get_zonal_average_fields(state, data, forcing, geom)
    _, data = O.get_shortwave_rad_fluxes(state, data, params, forcing, geom)
    return key, data


def test_shortwave_radiation(goldens, params):
    key, data = _sw_case(goldens, params)
    sw = data.shortwave_rad
    np.testing.assert_allclose(sw.rsds[0, :], goldens[key + "2"], atol=1e-4)
    assert np.allclose(sw.rsns[0, :], goldens[key + "3"], atol=1e-4)
    assert np.allclose(sw.ftop[0, :], goldens[key + "4"], atol=1e-4)
    assert np.allclose(np.mean(sw.dfabs, axis=0)[0, :], goldens[key + "5"], atol=1e-4)
    assert np.allclose(np.mean(sw.dfabs, axis=2)[:, 0], goldens[key + "6"], atol=1e-4)


def _tyear(days_since_1970, seconds=0.0):
    """fraction_of_year_elapsed (date.py:59-77) for a day count since 1970-01-01."""
    d = np.floor(days_since_1970 % O.DAYS_YEAR) + seconds / 86400.0
    return np.float32(d / O.DAYS_YEAR)


def test_zonal_fields_properties(params, geom):
    """test_output_shapes / test_solar_radiation_values / test_polar_night_cooling /
    test_ozone_absorption / test_random_input_consistency (shortwave_radiation_test.py:227-305).
    Dates: 2000-03-21 is day 11037 since 1970-01-01, 2000-04-01 12:00 is day 11048 + 12 h."""
    state = O.make_state(ZXY)
    for ty in (_tyear(11037), _tyear(11048, 43200.0)):
        data = O.get_zonal_average_fields(state, O.zeros_data(XY, KX, O.make_date(tyear=ty)),
                                          None, geom)
        sw = data.shortwave_rad
        for f in (sw.fsol, sw.ozupp, sw.ozone, sw.stratz, sw.zenit):
            assert f.shape == XY and np.all(f >= 0)
        assert np.allclose(sw.fsol[:, 0], O.solar(ty, geometry=geom)[0])
        assert np.all(np.maximum(6.0 - sw.fsol, 0) == sw.stratz)
    flat2 = 1.5 * geom.sia ** 2 - 0.5
    exp_oz = 0.4 * O.EPSSW * (1.0 + max(0.0, np.cos(4.0 * np.arcsin(1.0) * (ty + 10.0 / 365.0)))
                              + 1.8 * flat2)
    np.testing.assert_allclose(sw.ozone[:, 0], sw.fsol[:, 0] * exp_oz[0], atol=1e-4)


def test_cloud_top_level_set_matches_advanced_indexing(params):
    """Lines 62-68 of shortwave_radiation.py: the literal advanced-indexing scatter equals the
    level-set form (whole planes written at every level that is any column's icltop)."""
    rng = np.random.default_rng(3)
    ix, il, kx = 6, 4, 8
    geom = O.make_geometry(ix, il, kx)
    state = O.make_state((kx, ix, il), specific_humidity=rng.uniform(0, 10, (kx, ix, il)),
                         normalized_surface_pressure=rng.uniform(0.9, 1.1, (ix, il)))
    data = O.zeros_data((ix, il), kx, O.make_date(tyear=0.3))
    data = O.get_zonal_average_fields(state, data, None, geom)
    sw = data.shortwave_rad
    sw.icltop = rng.integers(1, kx + 1, (ix, il))
    sw.cloudc = rng.uniform(0, 1, (ix, il)).astype(F32)
    sw.cloudstr = rng.uniform(0, 0.5, (ix, il)).astype(F32)
    sw.qcloud = rng.uniform(0, 5, (ix, il)).astype(F32)
    data.mod_radcon.albsfc = rng.uniform(0, 0.5, (ix, il)).astype(F32)
    t1, d1 = O.shortwave_rad_fluxes(state, data, params, None, geom, literal_scatter=True)
    t2, d2 = O.shortwave_rad_fluxes(state, data, params, None, geom, literal_scatter=False)
    for a, b in ((d1.shortwave_rad.dfabs, d2.shortwave_rad.dfabs),
                 (d1.shortwave_rad.rsds, d2.shortwave_rad.rsds),
                 (d1.mod_radcon.flux, d2.mod_radcon.flux), (t1.temperature, t2.temperature)):
        np.testing.assert_array_equal(a, b)
    # and the effect is real: a column's result depends on other columns' icltop
    sw.icltop = np.full((ix, il), kx - 2)
    sw.icltop[0, 0] = 2
    _, d3 = O.shortwave_rad_fluxes(state, data, params, None, geom)
    sw.icltop[0, 0] = kx - 2
    _, d4 = O.shortwave_rad_fluxes(state, data, params, None, geom)
    assert not np.allclose(d3.shortwave_rad.rsds[1:], d4.shortwave_rad.rsds[1:])


# ---- longwave_radiation_test.py -----------------------------------------------------------
def test_downward_longwave(goldens, params, geom):
    key = "longwave_radiation_test::test_downward_longwave_rad_fluxes::"
    n = IX * IL * KX
    step = (250.0 - 130.0) / (n - 1)
    ta = (F32(130.0) + F32(step) * np.arange(n, dtype=F32)).reshape(KX, IL, IX).transpose(0, 2, 1)
    state = O.make_state(ZXY, temperature=ta)
    _, data = O.get_downward_longwave_rad_fluxes(state, O.zeros_data(XY, KX, O.make_date()),
                                                 params, None, geom)
    assert np.allclose(data.surface_flux.rlds[:5, :5], goldens[key + "0"], atol=1e-4)
    assert np.allclose(data.longwave_rad.dfabs[:, 0, 0], goldens[key + "1"], atol=1e-4)
    assert np.allclose(np.mean(data.mod_radcon.st4a[:, :5, :5, :], axis=0), goldens[key + "2"],
                       atol=1e-4)


def test_upward_longwave(goldens, params, geom):
    key = "longwave_radiation_test::test_upward_longwave_rad_fluxes::"
    data = O.zeros_data(XY, KX, O.make_date())
    data.longwave_rad.dfabs = np.ones(ZXY, F32)
    data.mod_radcon.st4a = np.ones(ZXY + (2,), F32)
    data.mod_radcon.flux = np.ones(XY + (4,), F32)
    data.mod_radcon.tau2 = (np.ones(ZXY + (4,), F32)
                            + np.arange(KX, dtype=F32)[:, None, None, None] * F32(0.1))
    data.mod_radcon.stratc = np.ones(XY + (2,), F32)
    data.surface_flux.rlus = np.zeros(XY + (3,), F32)
    data.surface_flux.rlus[:, :, 2] = 1.0
    data.surface_flux.rlds = np.ones(XY, F32)
    data.surface_flux.tsfc = np.ones(XY, F32) * 300
    state = O.make_state(ZXY, temperature=np.ones(ZXY, F32) * 300)
    _, out = O.get_upward_longwave_rad_fluxes(state, data, params, None, geom)
    assert abs(out.surface_flux.rlns[0, 0] - goldens[key + "assign::fsfc_f90"]) <= 1e-5
    assert abs(out.longwave_rad.ftop[0, 0] - goldens[key + "assign::ftop_f90"]) <= 1e-5 + 1e-8 * 2.04
    assert np.allclose(out.longwave_rad.dfabs[:, 0, 0], goldens[key + "0"], atol=1e-5)
    assert np.allclose(out.mod_radcon.flux[0, 0, :], goldens[key + "1"], atol=1e-5)


# ---- surface_flux_test.py -----------------------------------------------------------------
def _sflux_case(params, ta, phi0, sst, forcing_fill):
    psa = np.ones(XY, F32)
    ua = va = np.ones(ZXY, F32)
    qa = F32(5.0) * np.ones(ZXY, F32)
    rh = F32(0.8) * np.ones(ZXY, F32)
    phi = F32(5000.0) * np.ones(ZXY, F32)
    geom = O.make_geometry(IX, IL, KX, lat="speedy", orog=np.float32(phi0) / F32(O.GRAV),
                           fmask=0.5)
    geom.phis0 = np.full(XY, F32(phi0))
    forcing = O.make_forcing(XY, fill=forcing_fill, lfluxland=True,
                             sea_surface_temperature=sst, soilw_am=0.5, stl_am=288.0)
    state = O.make_state(ZXY, u_wind=ua, v_wind=va, temperature=ta * np.ones(ZXY, F32),
                         specific_humidity=qa, geopotential=phi, normalized_surface_pressure=psa)
    data = O.zeros_data(XY, KX, O.make_date())
    data.surface_flux.rlds = F32(400.0) * np.ones(XY, F32)
    data.humidity.rh = rh
    data.shortwave_rad.rsds = F32(400.0) * np.ones(XY, F32)
    return O.get_surface_fluxes(state, data, params, forcing, geom)


@pytest.mark.parametrize("case,ta,phi0", [(1, 288.0, 500.0), (2, 288.0, 500.0), (3, 288.0, -10.0),
                                          (4, 300.0, 500.0), (5, 285.0, 500.0)])
def test_surface_fluxes_cases(goldens, params, case, ta, phi0):
    _, data = _sflux_case(params, F32(ta), phi0, 290.0, 0.0)
    s = data.surface_flux
    vars_ = [s.ustr, s.vstr, s.shf, s.evap, s.rlus, s.hfluxn, s.tsfc, s.tskin, s.u0, s.v0, s.t0]
    got = np.array([[np.max(v), np.min(v), np.mean(v)] for v in vars_])
    want = goldens[f"surface_flux_test::test_surface_fluxes_test{case}::0"].T
    assert np.allclose(got, want, rtol=2e-5)


def test_updated_surface_flux(goldens, params):
    key = "surface_flux_test::test_updated_surface_flux::"
    xy, zxy = XY, ZXY
    psa = np.ones(xy, F32)
    ta = np.ones(zxy, F32) * 290
    qa = np.ones(zxy, F32)
    rh = np.ones(zxy, F32) * F32(0.5)
    phi = np.ones(zxy, F32) * np.arange(KX)[::-1][:, None, None].astype(F32)
    geom = O.make_geometry(IX, IL, KX, lat="speedy", orog=0.0, fmask=0.5)
    forcing = O.make_forcing(xy, fill=1.0, lfluxland=True, sea_surface_temperature=292.0,
                             soilw_am=0.5, stl_am=288.0)
    state = O.make_state(zxy, u_wind=np.ones(zxy), v_wind=np.ones(zxy), temperature=ta,
                         specific_humidity=qa, geopotential=phi, normalized_surface_pressure=psa)
    data = O.zeros_data(xy, KX, O.make_date())
    data.surface_flux.rlds = F32(400) * np.ones(xy, F32)
    data.humidity.rh = rh
    data.shortwave_rad.rsds = F32(400) * np.ones(xy, F32)
    _, data = O.get_surface_fluxes(state, data, params, forcing, geom)
    s = data.surface_flux
    for n, f in enumerate([s.ustr, s.vstr, s.shf, s.evap, s.rlus, s.hfluxn]):
        assert np.allclose(f[0, 0, :], goldens[key + str(n)], atol=1e-4), n
    fl = goldens[key + "floats"]
    assert np.isclose(s.tsfc[0, 0], fl[26], atol=1e-4)
    assert np.isclose(s.tskin[0, 0], fl[28], atol=1e-4)
    assert np.isclose(s.u0[0, 0], fl[30], atol=1e-4)
    assert np.isclose(s.v0[0, 0], fl[32], atol=1e-4)
    assert np.isclose(s.t0[0, 0], fl[34], atol=1e-4)


def test_surface_drag(goldens, params):
    forog = O.get_orog_land_sfc_drag(F32(500.0) * np.ones(XY, F32), params.surface_flux.hdrag)
    want = goldens["surface_flux_test::test_surface_fluxes_drag_test::0"]
    assert round(float(np.max(forog)) - want[0], 7) == 0
    assert round(float(np.min(forog)) - want[1], 7) == 0


# ---- vertical_diffusion_test.py -----------------------------------------------------------
def test_vertical_diffusion(goldens, params):
    key = "vertical_diffusion_test::test_get_vertical_diffusion_tend::"
    xy, zxy = (1, 1), (KX, 1, 1)
    geom1 = O.make_geometry(1, 1, KX, lat=[0.0])
    b = lambda a: np.ones(xy, F32) * np.asarray(a, F32)[:, None, None]
    se = b(np.linspace(400, 300, KX, dtype=F32))
    rh = b(np.linspace(0.1, 0.9, KX, dtype=F32))
    qa, qsat = b(goldens[key + "0"]), b(goldens[key + "1"])
    phi = b(np.linspace(150000, 0, KX, dtype=F32))
    data = O.zeros_data(xy, KX, O.make_date())
    data.humidity.rh, data.humidity.qsat = rh, qsat
    data.convection.iptop, data.convection.se = np.ones(xy, np.int64), se
    state = O.make_state(zxy, specific_humidity=qa, geopotential=phi)
    tend, _ = O.get_vertical_diffusion_tend(state, data, params, None, geom1)
    assert np.allclose(tend.u_wind, 0, atol=1e-9) and np.allclose(tend.v_wind, 0, atol=1e-9)
    assert np.allclose(tend.temperature[:, 0, 0], goldens[key + "2"], atol=1e-9)
    assert np.allclose(tend.specific_humidity[:, 0, 0], goldens[key + "3"], atol=1e-9)


# ---- humidity_test.py (property tests) ----------------------------------------------------
def test_humidity_properties(params, geom):
    temp = np.ones(ZXY, F32) * 273
    pressure = np.ones(XY, F32)
    sigma = 4
    qs = O.get_qsat(temp[sigma], pressure, F32(sigma))
    assert np.all(qs >= 0)
    for t in (100.0, 350.0):
        assert np.all(O.get_qsat(np.ones(XY, F32) * F32(t), pressure, F32(sigma)) >= 0)
    data = O.zeros_data(XY, KX, O.make_date())
    st = O.make_state(ZXY, temperature=temp, specific_humidity=np.zeros(ZXY),
                      normalized_surface_pressure=pressure)
    _, d = O.spec_hum_to_rel_hum(st, data, params, None, geom)
    assert np.all(d.humidity.rh == 0)
    st = O.make_state(ZXY, temperature=np.ones(ZXY) * 400, specific_humidity=np.zeros(ZXY),
                      normalized_surface_pressure=pressure * 10)
    _, d = O.spec_hum_to_rel_hum(st, data, params, None, geom)
    assert np.all((d.humidity.rh >= 0) & (d.humidity.rh <= 1))
    st = O.make_state(ZXY, temperature=temp, specific_humidity=np.ones(ZXY) * 2,
                      normalized_surface_pressure=pressure)
    _, d = O.spec_hum_to_rel_hum(st, data, params, None, geom)
    qa, _ = O.rel_hum_to_spec_hum(temp[0], pressure, geom.fsg[0], d.humidity.rh[0])
    assert np.allclose(qa, 2.0, atol=1e-6)
    qg = np.ones(ZXY, F32) * (d.humidity.qsat[:, 0, 0][:, None, None] - F32(1e-6))
    st.specific_humidity = qg
    _, d2 = O.spec_hum_to_rel_hum(st, data, params, None, geom)
    assert np.all(d2.humidity.rh >= 0.99) and np.all(d2.humidity.rh <= 1)


# ---- speedy_physics_test.py ---------------------------------------------------------------
def test_speedy_single_column_smoke(params):
    shape = (8, 1, 1)
    geom1 = O.make_geometry(1, 1, 8, lat=[0.0])
    tend, data = O.compute_tendencies(O.make_state(shape), O.make_forcing((1, 1), fill=1.0),
                                      geom1, O.make_date(), params)
    assert tend is not None and data is not None


def test_full_chain_finite_on_config0_like_state(params):
    import importlib
    synthetic = importlib.import_module("jax-gcm_b200").synthetic
    case = synthetic.config0_instance(seed=0, ix=32, il=16, lfluxland=True)
    tend, data = O.physics_step(*case.oracle_args(params))
    for f in (tend.u_wind, tend.v_wind, tend.temperature, tend.specific_humidity):
        assert np.all(np.isfinite(f))
    assert np.any(tend.temperature != 0)


# ---- orographic correction (orographic_correction_test.py) ----------------------------------
ORO = "orographic_correction_test::test_speedy_fortran_numerical_equivalence::"


def test_orographic_profiles_match_fortran(goldens):
    """test_speedy_fortran_numerical_equivalence (orographic_correction_test.py:279-333): the
    vertical profiles at 8 levels and the horizontal temperature correction of a 4x4
    orography against SPEEDY Fortran output, with the reference's tolerances."""
    _, fsg, *_ = O.vertical_tables(8)
    tcorv, qcorv = O.orographic_vertical_profiles(fsg)
    np.testing.assert_allclose(tcorv, g(goldens, ORO + "1"), rtol=1e-3, atol=1e-6)
    np.testing.assert_allclose(qcorv, g(goldens, ORO + "2"), rtol=1e-3, atol=1e-12)
    orog = g(goldens, ORO + "0").astype(F32)
    phis0 = (F32(O.GRAV) * orog).astype(F32)
    ones = np.ones_like(phis0)
    tcorh, _ = O.orographic_horizontal(phis0, ones, ones * F32(288.0), ones * F32(285.0))
    np.testing.assert_allclose(tcorh, g(goldens, ORO + "3"), rtol=1e-3, atol=1e-12)
    assert tcorv[0] == 0.0 and np.all(tcorv[1:] > 0.0) and np.all(tcorv < 1.0)
    assert qcorv[0] == 0.0 and qcorv[1] == 0.0 and np.all(qcorv[2:] > 0.0)


def test_orographic_tendencies_properties():
    """test_humidity_horizontal_correction and test_get_orographic_correction_tendencies
    (orographic_correction_test.py:162-222): on the reference's test setup (Gaussian 1000 m
    mountain, 70 % land, SST 285 K, land 288 K) the humidity correction is non-zero and bounded,
    the wind tendencies are zero and the temperature and humidity tendencies are bounded; the
    tendencies times the step equal the corrections applied to the state (lines 224-257)."""
    ix, il = 96, 48
    li, lj = np.meshgrid(np.arange(ix), np.arange(il), indexing="ij")
    orog = (1000.0 * np.exp(-((li - ix // 2) ** 2 / (2 * (ix / 8) ** 2) +
                              (lj - il // 2) ** 2 / (2 * (il / 8) ** 2)))).astype(F32)
    geom = O.make_geometry(ix, il, 8, orog=orog, fmask=np.full((ix, il), 0.7, F32))
    fo = O.make_forcing((ix, il), sea_surface_temperature=np.full((ix, il), 285.0, F32),
                        stl_am=np.full((ix, il), 288.0, F32))
    _, qcorh = O.orographic_horizontal(geom.phis0, geom.fmask, fo.stl_am,
                                       fo.sea_surface_temperature)
    assert np.all(np.abs(qcorh) < 10.0) and np.any(qcorh != 0.0)
    st = O.make_state((8, ix, il))
    data = O.zeros_data((ix, il), 8, O.make_date())
    t, _ = O.get_orographic_correction_tendencies(st, data, O.default_parameters(),
                                                  O.forcing_day_slice(fo, data.date), geom)
    assert np.all(t.u_wind == 0.0) and np.all(t.v_wind == 0.0)
    assert np.any(t.temperature != 0.0) and np.any(t.specific_humidity != 0.0)
    assert np.all(np.abs(t.temperature) < 0.05) and np.all(np.abs(t.specific_humidity) < 0.01)
    tcorv, qcorv = O.orographic_vertical_profiles(geom.fsg)
    tcorh, _ = O.orographic_horizontal(geom.phis0, geom.fmask, fo.stl_am,
                                       fo.sea_surface_temperature)
    np.testing.assert_allclose(t.temperature * data.date.dt_seconds,
                               tcorh[None] * tcorv[:, None, None], rtol=1e-4, atol=2e-5)
