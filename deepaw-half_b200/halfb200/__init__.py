"""Python binding of the B200 libhalf (ctypes over the C ABI in include/half.h).

The library itself is C/C++/CUDA (deepaw-half_b200/csrc, built into
deepaw-half_b200/lib/libhalf.so); this package only marshals arguments.
Import it before torch when both are used in one process, so that the CUDA
toolkit's cuBLAS (with FP32 tensor-core emulation) is the one the process
binds first.
"""
from .lib import (HalfError, Context, load_library, library_path, abi_version, version_string, capabilities,
                  occupations, tc_cgemm, allocation_counts,
                  HALF_SUCCESS, HALF_ERROR_INVALID_ARGUMENT, HALF_ERROR_IO, HALF_ERROR_INVALID_HANDLE,
                  HALF_ERROR_CAPACITY, HALF_ERROR_UNAVAILABLE, HALF_ERROR_INTERNAL, XC, BACKEND, SOLVER, PRECISION)

__all__ = ["HalfError", "Context", "load_library", "library_path", "abi_version", "version_string", "capabilities",
           "occupations", "tc_cgemm", "allocation_counts",
           "HALF_SUCCESS", "HALF_ERROR_INVALID_ARGUMENT", "HALF_ERROR_IO", "HALF_ERROR_INVALID_HANDLE",
           "HALF_ERROR_CAPACITY", "HALF_ERROR_UNAVAILABLE", "HALF_ERROR_INTERNAL", "XC", "BACKEND", "SOLVER",
           "PRECISION"]
