"""perix_b200: B200-native (sm_100a) backend for PeriX's PDDO hot path.

The compute path is ``libperix_b200.so`` (C++20 host + hand-written CUDA kernels) behind the C-ABI declared in
``include/perix_b200.h``; this package is a thin ctypes mirror of that ABI for Python callers, tests and the
bench.  It never computes on the CPU: if the library is missing, or no GPU is present, the call fails with
``PxbError``.
"""
from .api import (PxbError, Context, lib, lib_path, lattice, families, families_vh, variable_horizon,  # noqa: F401
                  crack_cut_mask, csr_pattern, multi_indices, elastic_constants, critical_stretch, FP64, MIXED, BC)

__all__ = ["PxbError", "Context", "lib", "lib_path", "lattice", "families", "families_vh", "variable_horizon",
           "crack_cut_mask", "csr_pattern", "multi_indices", "elastic_constants", "critical_stretch", "FP64", "MIXED",
           "BC"]
