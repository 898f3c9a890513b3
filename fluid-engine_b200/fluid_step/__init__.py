"""fluid_step — host side of the B200-native DFSPH step.

The compute path is libfluidstep.so (hand-written sm_100a CUDA behind the C
ABI of include/fluid_step.h).  This package loads it and mirrors the
reference's host interface: `SimulationParams`, `GpuPhysicsData`, the
`ComputeStep` passes and the `ComputePipelines` registry
(src/renderer/pipelines/mod.rs:52-124).
"""
from . import _abi, scene  # noqa: F401
from ._abi import (FE_MODE_FIXED, FE_MODE_REFERENCE, FE_SOLVER_FIXED_ITERS,  # noqa: F401
                   FE_SOLVER_TOLERANCE, FE_SORT_BITONIC, FE_SORT_RADIX, FeParams,
                   FeStats, FluidStepError, LibraryMissing, default_params,
                   load_library)
