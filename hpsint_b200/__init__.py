"""hpsint_b200: B200-native matrix-free sintering operator.

The CUDA kernels and the C ABI live in csrc/ (built into libhpsint_b200.so);
this package is the host-side mirror of hpsint's operator interface.
"""
from .operator import (BlockPreconditioner2, DampedNewtonSolver, HostJvpPipeline, Mesh, NewtonStatistics,
                       NonLinearData, Params, SinteringOperatorGeneric, bdf_weights)
from ._lib import SintError, kernel_launch_count

__all__ = ["Mesh", "Params", "SinteringOperatorGeneric", "BlockPreconditioner2", "DampedNewtonSolver",
           "NonLinearData", "NewtonStatistics", "HostJvpPipeline", "bdf_weights", "SintError", "kernel_launch_count"]
