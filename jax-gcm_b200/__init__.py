"""B200-native (sm_100a) SPEEDY column physics with the interface of JAX-GCM's physics package.

Import name: the package directory is ``jax-gcm_b200``; load it with
``importlib.import_module("jax-gcm_b200")`` (the hyphen rules out a plain ``import``).
"""
from . import _lib, synthetic  # noqa: F401
from .batched import Ensemble, Member  # noqa: F401
from . import serving  # noqa: F401
from . import adjoint, held_suarez, rollout  # noqa: F401
from .held_suarez import HeldSuarezPhysics  # noqa: F401
from .physics import (DateData, ForcingData, Geometry, Parameters, Physics,  # noqa: F401
                      PhysicsState, PhysicsTendency, SpeedyPhysics,
                      get_physical_tendencies_columns, instance_to_device)

__all__ = ["Ensemble", "Member", "HeldSuarezPhysics", "DateData", "ForcingData", "Geometry", "Parameters", "Physics", "PhysicsState",
           "PhysicsTendency", "SpeedyPhysics", "get_physical_tendencies_columns", "synthetic"]
