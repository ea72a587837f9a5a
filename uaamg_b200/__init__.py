"""B200-native UAAMG-preconditioned CG pressure solver.

The compute path is ``libuaamg_b200.so`` (hand-written sm_100a CUDA behind the
C-ABI of ``include/uaamg.h``); this package is its host-side mirror of the
reference's solver surface (Grid/Grid3D, Solver, Factory, PressureProjection).
"""
from . import _capi  # noqa: F401
from .solver import (  # noqa: F401
    Factory,
    Factory3D,
    GpuUAAMGPCG,
    GpuUAAMGPCG3D,
    Grid,
    Grid3D,
    Handle,
    PressureProjection,
    PressureProjection3D,
    Solver,
    Solver3D,
    SolverKind,
)

__all__ = [
    "Factory", "Factory3D", "GpuUAAMGPCG", "GpuUAAMGPCG3D", "Grid", "Grid3D", "Handle",
    "PressureProjection", "PressureProjection3D", "Solver", "Solver3D", "SolverKind",
]
