"""spmv_b200: libspmv's hot path (Matrix mult/transpmult, L2GMap
update/reverse_update, cg) as hand-written sm_100a CUDA kernels behind a C ABI.

The native library is built in-tree by ``python -m spmv_b200.build``; importing
the package does not build or load anything, and every compute call fails
loudly if ``libspmv_b200.so`` is missing (there is no CPU fallback).
"""
from ._lib import SpmvError  # noqa: F401
from .core import (Comm, L2GMap, Matrix, cg, cg_mixed, create_matrix,  # noqa: F401
                   owner_ranges, read_petsc_binary, read_petsc_binary_vector)

__all__ = ["Comm", "L2GMap", "Matrix", "cg", "cg_mixed", "create_matrix", "SpmvError",
           "owner_ranges", "read_petsc_binary", "read_petsc_binary_vector"]
