"""B200-native UAAMG-preconditioned CG pressure solver.

The compute path is ``libuaamg_b200.so`` (hand-written sm_100a CUDA behind the
C-ABI of ``include/uaamg.h``); this package is its host-side mirror of the
reference's solver surface (Grid/Grid3D, Solver, Factory, PressureProjection).

Batched and served solves run many CUDA streams at once; the device's default of
8 hardware work queues would make unrelated streams wait on one another, so 32
queues are requested before the process creates its CUDA context (an explicit
CUDA_DEVICE_MAX_CONNECTIONS wins).
"""
import os as _os

_os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

from . import _capi  # noqa: F401,E402
from .solver import (  # noqa: F401,E402
    Factory,
    Factory3D,
    GpuUAAMGPCG,
    GpuUAAMGPCG3D,
    Grid,
    Grid3D,
    Handle,
    Server,
    PressureProjection,
    PressureProjection3D,
    Solver,
    Solver3D,
    SolverKind,
)

__all__ = [
    "Factory", "Factory3D", "GpuUAAMGPCG", "GpuUAAMGPCG3D", "Grid", "Grid3D", "Handle", "Server",
    "PressureProjection", "PressureProjection3D", "Solver", "Solver3D", "SolverKind",
]
