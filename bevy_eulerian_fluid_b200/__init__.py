"""B200-native per-step Eulerian fluid hot path behind the bevy_eulerian_fluid plugin API.

The compute path is libefl_b200.so (hand-written sm_100a kernels behind the
C ABI of include/efl.h).  Importing this package does not load the library;
the first simulation does, and fails loudly if the library is missing.
"""
from . import _capi as capi  # noqa: F401
from .plugin import (  # noqa: F401
    Collider, FastIterativeMethodConfig, Fluid, FluidPlugin, FluidSettings, FluidSource, FluidSourceMode,
    FluidSourceOneshot, FluidSourceShape, FluidSourceVelocity, FluidStatus, FluidTextures, FluidToSolidForce,
    ForcesToFluid, ForceToFluid, GaussSeidelConfig, LevelsetParticles, LocalForces, MultiGridConfig,
    ParticleLevelsetTwoLayersPlugin, ProjectionMethod, ReinitializeMethod, RigidBody, RigidBodyKind,
)

__all__ = [
    "capi", "Collider", "FastIterativeMethodConfig", "Fluid", "FluidPlugin", "FluidSettings", "FluidSource",
    "FluidSourceMode", "FluidSourceOneshot", "FluidSourceShape", "FluidSourceVelocity", "FluidStatus",
    "FluidTextures", "FluidToSolidForce", "ForcesToFluid", "ForceToFluid", "GaussSeidelConfig", "LevelsetParticles",
    "LocalForces", "MultiGridConfig", "ParticleLevelsetTwoLayersPlugin", "ProjectionMethod", "ReinitializeMethod",
    "RigidBody", "RigidBodyKind",
]
