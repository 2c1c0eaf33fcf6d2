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
__all__ = ["VoxelPlateModel", "VoxelPlateExModel", "VoxelTuringModel", "VoxelArrayModel",
           "TuringPattern"]


def __getattr__(name):
    # imported on first use, so that ``python -m pymonteopt_b200.turing`` runs
    # the module once rather than over an already imported copy
    if name == "TuringPattern":
        from .turing import TuringPattern
        return TuringPattern
    raise AttributeError(f"module {__name__!r} has no attribute {name!r}")
