"""How close two float32 evaluations of the reference arithmetic can be expected to agree,
element by element: the float32 oracle against itself with every exponential's result moved by
a seeded relative noise of up to 2 ulps (Monte Carlo arithmetic on the one operation whose last
bits differ between float32 math libraries; oracle.speedy_oracle.perturbed_exp).

The temperature and humidity tendencies and the convective precipitation are sums of terms that
cancel, so a last-bit change of one exponential moves small elements of these fields by far more
than 1e-5 of their own size.  The smallest per-field floor at which the two evaluations still
agree within 1e-5 elementwise is a large fraction of the field's maximum, so the parity bar's
floors for these fields (tests/helpers.py ELEM_FLOOR) cannot be small; the winds and the
large-scale precipitation are not sensitive.  This test pins both statements on the oracle
alone (no GPU)."""
import importlib

import numpy as np
import pytest

from oracle import speedy_oracle as O
from tests import helpers as H


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


def twin_floors(inst, seeds=(7, 8)):
    args = list(H.oracle_args(inst))
    ref = H.oracle_fields(*O.compute_tendencies(*args))
    worst = {}
    for s in seeds:
        with O.perturbed_exp(seed=s, ulps=2.0):
            got = H.oracle_fields(*O.compute_tendencies(*args))
        for k in H.STRICT_FIELDS:
            worst[k] = max(worst.get(k, 0.0), H.required_floor(got[k], ref[k]))
    return worst


@pytest.mark.parametrize("case", ["t31_aquaplanet", "t85_land_16"])
def test_exponential_last_bits_set_the_elementwise_floor(pkg, case):
    if case == "t31_aquaplanet":
        inst = pkg.synthetic.config0_instance(seed=11, lfluxland=True)
    else:
        inst = pkg.synthetic.land_instance(85, 256, 128, 16, sst_noise=1.5)
    f = twin_floors(inst)
    print(case, {k: round(v, 3) for k, v in f.items()})
    # a floor of 1e-3 of the maximum would fail the reference arithmetic against itself
    assert f["temperature"] > 0.05 and f["specific_humidity"] > 0.005
    # the parity bar's floors admit it
    for k, v in f.items():
        assert v <= H.ELEM_FLOOR[k], (k, v, H.ELEM_FLOOR[k])
    assert f["u_wind"] <= 1e-3 and f["v_wind"] <= 1e-3 and f["precls"] <= 1e-3
