"""Writers for PETSc binary files (the format spmv::read_petsc_binary and
read_petsc_binary_vector read, read_petsc.cpp:32-260): big-endian int32
{1211216, nrows, ncols, nnz}, row lengths, column indices, float64 values;
vectors {1211214, n} then float64 values.  For preparing inputs (PETSc writes
the same files with -ksp_view_mat binary / -ksp_view_rhs binary)."""
from __future__ import annotations

import numpy as np


def write_matrix(filename, rowptr, colind, values, ncols: int) -> None:
    """Writes a global CSR matrix (int row pointers, column indices in file
    order per row, float64 values)."""
    rowptr = np.asarray(rowptr, dtype=np.int64)
    nrows = len(rowptr) - 1
    nnz = int(rowptr[-1])
    lens = np.diff(rowptr)
    with open(filename, "wb") as f:
        f.write(np.array([1211216, nrows, int(ncols), nnz], dtype=">i4").tobytes())
        f.write(lens.astype(">i4").tobytes())
        f.write(np.asarray(colind[:nnz]).astype(">i4").tobytes())
        f.write(np.asarray(values[:nnz], dtype=np.float64).astype(">f8").tobytes())


def write_vector(filename, values) -> None:
    values = np.asarray(values, dtype=np.float64)
    with open(filename, "wb") as f:
        f.write(np.array([1211214, len(values)], dtype=">i4").tobytes())
        f.write(values.astype(">f8").tobytes())
