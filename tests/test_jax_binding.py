"""The JAX side of the drop-in (jax-gcm_b200/jax_physics.py, jax_binding/spd_ffi.cc): where
jax, its FFI headers and the reference package are importable, a one-day Model run with
SpeedyPhysicsB200 swapped in (jcm/model.py:171) against the same run with the reference's
SpeedyPhysics: global means of temperature and humidity and the day's precipitation within
1e-3 relative, and a jax.grad through the FFI call.  Skipped where they are not (this image
has no jax)."""
import importlib

import numpy as np
import pytest

jax = pytest.importorskip("jax")
jcm_model = pytest.importorskip("jcm.model")


@pytest.fixture(scope="module")
def physics_b200():
    jp = importlib.import_module("jax-gcm_b200.jax_physics")
    try:
        jp.build_ffi()
    except (ImportError, OSError) as e:
        pytest.skip(f"jax FFI headers unavailable: {e}")
    return jp.SpeedyPhysicsB200()


@pytest.mark.gpu
def test_one_day_model_run_matches_reference_means(physics_b200):
    from jcm.model import Model
    from jcm.physics.speedy.speedy_physics import SpeedyPhysics
    ref = Model(time_step=30.0, layers=8, horizontal_resolution=31, physics=SpeedyPhysics())
    b200 = Model(time_step=30.0, layers=8, horizontal_resolution=31, physics=physics_b200)
    out_ref = ref.run(total_time=1.0, save_interval=1.0)
    out_b200 = b200.run(total_time=1.0, save_interval=1.0)
    for name in ("temperature", "specific_humidity"):
        a = np.asarray(getattr(out_ref.dynamics, name)).mean()
        b = np.asarray(getattr(out_b200.dynamics, name)).mean()
        assert abs(b - a) <= 1e-3 * abs(a), name
    pa = np.asarray(out_ref.physics.convection.precnv + out_ref.physics.condensation.precls).mean()
    pb = np.asarray(out_b200.physics.convection.precnv + out_b200.physics.condensation.precls).mean()
    assert abs(pb - pa) <= 1e-3 * abs(pa)


@pytest.mark.gpu
def test_grad_flows_through_the_ffi_call(physics_b200):
    import jax.numpy as jnp
    from jcm.geometry import Geometry
    from jcm.physics_interface import PhysicsState
    from jcm.forcing import ForcingData
    from jcm.date import DateData
    geo = Geometry.from_grid_shape((96, 48), 8)
    st = PhysicsState.ones((8, 96, 48))
    st = st.copy(temperature=st.temperature * 280.0, specific_humidity=st.specific_humidity * 2.0)
    fo = ForcingData.ones((96, 48))
    da = DateData.zeros()

    def loss(t):
        tend, _ = physics_b200.compute_tendencies(st.copy(temperature=t), fo, geo, da)
        return jnp.sum(tend.temperature)

    g = jax.grad(loss)(st.temperature)
    assert np.all(np.isfinite(np.asarray(g)))
