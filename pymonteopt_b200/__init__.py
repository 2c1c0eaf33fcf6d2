"""pymonteopt_b200 — B200-native voxel Monte Carlo photon transport.

A drop-in for the transport path of pyMonteOpt (``pymopt.voxel_gpu``): the
same model classes, params keys and result getters, computed by hand-written
sm_100a CUDA kernels behind a C ABI (``include/pmo_b200.h``).
"""
__version__ = "0.1.0"

from .voxel import (  # noqa: E402,F401
    VoxelArrayModel,
    VoxelPlateExModel,
    VoxelPlateModel,
    VoxelTuringModel,
)
from .turing import TuringPattern  # noqa: E402,F401

__all__ = ["VoxelPlateModel", "VoxelPlateExModel", "VoxelTuringModel", "VoxelArrayModel",
           "TuringPattern"]
