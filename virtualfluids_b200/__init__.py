"""B200-native implementation of the VirtualFluids GPU time-step hot path.

D3Q27 K17 cumulant collision with in-place esoteric-twist streaming, the bounce-back,
interpolated, velocity and non-equilibrium pressure boundary kernels, the interpolation between
refinement levels and the FP64 reductions,
as hand-written sm_100a CUDA behind the C ABI of ``include/vfb.h`` (``libvfb.so``). This package
is the Python host side: set-up objects mirroring the reference's Parameter /
BoundaryConditionFactory / Simulation, a builder for levels in the reference layout, and
structured boxes. The native library is loaded on first use (``lib()``) and a missing or stale
library raises there; there is no fallback.
"""
from . import _native
from ._native import VfbError, lib
from .box import Box
from .grid import Interface, ListGrid, MultiLevelGrid, refine_box
from .pool import Pool
from .simulation import (BoundaryConditionFactory, GridScalingFactory, InterpolationCells, K17ParameterWarning,
                         Parameter, Simulation, scale_coarse_to_fine, scale_fine_to_coarse)

__all__ = ["Box", "BoundaryConditionFactory", "GridScalingFactory", "Interface", "InterpolationCells",
           "K17ParameterWarning", "ListGrid",
           "MultiLevelGrid", "Parameter", "Pool", "Simulation", "VfbError", "lib", "refine_box", "scale_coarse_to_fine",
           "scale_fine_to_coarse", "_native"]
