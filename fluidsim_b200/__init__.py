"""UniformCUDA: a B200-native backend for FluidSim's uniform MAC-grid projection.

The product is libfluidcuda.so (hand-written sm_100a kernels behind the C ABI in
include/fluidcuda.h). This package is its Python host mirror of FluidSim's engine contract.
"""
from ._native import FluidCudaError, FluidInvalidArgument, FluidLifecycleError, kernel_launches, lib
from .grid import FluidGrid, FluidGridState, ProjectionBatch, ProjectionResult

__all__ = [
    "FluidGrid",
    "FluidGridState",
    "ProjectionBatch",
    "ProjectionResult",
    "FluidCudaError",
    "FluidInvalidArgument",
    "FluidLifecycleError",
    "kernel_launches",
    "lib",
]
