"""B200-native DG residual / time-step path for the 1D/2D gamma-model multifluid Euler solver.

The compute path is ``lib/libdgb.so`` (C++ host setup + sm_100a CUDA kernels) behind the C ABI in
``include/dgb.h``; this package is its Python binding.  There is no CPU fallback: device calls
fail when the library or the GPU is missing.
"""
from ._ffi import DGBError, RK4, SSPRK3  # noqa: F401
from .solver import DGBatch, DGSolver, Problem, write_msh  # noqa: F401

__all__ = ["DGBatch", "DGSolver", "Problem", "write_msh", "DGBError", "RK4", "SSPRK3"]
