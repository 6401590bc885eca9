"""felbm_gpu_b200 — B200-native Lee–Liu free-energy multiphase D3Q19 step.

The product is the native library ``_lib/libfelbm_b200.so`` (C-ABI in
include/felbm_b200.h: hand-written sm_100a kernels behind a C++ host engine).
This package is a thin Python mirror of the reference engine interface for
tests, benchmarks and scripting.
"""
from . import _capi  # noqa: F401  (raises ImportError if the library is missing)
from .engine import Batch, MultiPhaseGPU, OpenBoundary, default_params  # noqa: F401
from . import geometry  # noqa: F401

__all__ = ["Batch", "MultiPhaseGPU", "OpenBoundary", "default_params", "geometry"]
