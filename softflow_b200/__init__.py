"""softflow_b200 -- B200-native implementation of the SoftFlow per-timestep
hot path (D2Q9 lattice Boltzmann + immersed-boundary capsules + scalar
transport) behind the C ABI of include/softflow_gpu.h.

The compute runs in libsoftflow_b200.so (sm_100a CUDA kernels); this package
is the host-side mirror of the reference engine API.
"""
from .engine import (  # noqa: F401
    BoundaryType,
    CapsuleShape,
    ChannelBuilder,
    CollisionModel,
    Ensemble,
    FluidParams,
    MembraneModel,
    MembraneParams,
    RepulsionParams,
    ScalarParams,
    Simulation,
    SimulationParams,
    build_circle_capsule,
)
from ._lib import SoftFlowGpuError, lib as load_library  # noqa: F401

__all__ = [
    "BoundaryType", "CapsuleShape", "ChannelBuilder", "CollisionModel", "Ensemble", "FluidParams",
    "MembraneModel", "MembraneParams", "RepulsionParams", "ScalarParams", "Simulation",
    "SimulationParams", "SoftFlowGpuError", "build_circle_capsule", "load_library",
]
