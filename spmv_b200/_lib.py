"""ctypes binding of libspmv_b200.so (the C ABI in include/spmv_b200.h)."""
from __future__ import annotations

import ctypes as C
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libspmv_b200.so"

# spmv_status
SUCCESS = 0
ERROR_INVALID_ARGUMENT = 1
ERROR_CUDA = 2
ERROR_OUT_OF_MEMORY = 3
ERROR_NO_DEVICE = 4
ERROR_BREAKDOWN = 5
ERROR_NOT_SUPPORTED = 6
ERROR_INTERNAL = 7

# spmv_dtype
FLOAT64, FLOAT32, COMPLEX64, COMPLEX128 = 0, 1, 2, 3
# spmv_memory
MEMORY_HOST, MEMORY_DEVICE = 0, 1
# spmv_kernel
KERNEL_AUTO, KERNEL_VECTOR, KERNEL_MERGE, KERNEL_SELL, KERNEL_STAGED = 0, 1, 2, 3, 4
KERNEL_NAMES = {0: "auto", 1: "vector", 2: "merge", 3: "sell", 4: "staged"}
# spmv_pattern_field
PATTERN_FIELDS = {"neighbours": 0, "send_count": 1, "recv_count": 2,
                  "send_offset": 3, "recv_offset": 4, "indexbuf": 5}

MAX_PARTS = 64


class SpmvError(RuntimeError):
    """A failed libspmv_b200 call; str() is the library's message (the
    reference's std::runtime_error text where it has one)."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


class CgInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("status", C.c_int),
                ("rnorm0", C.c_double), ("rnorm", C.c_double)]


class IrInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int),
                ("status", C.c_int), ("converged", C.c_int), ("relres", C.c_double)]


BatchInfo = IrInfo  # same layout as spmv_batch_info


class BatchConfig(C.Structure):
    _fields_ = [("ctas_per_sm", C.c_int), ("tile_rows", C.c_int), ("rhs_lanes", C.c_int),
                ("window", C.c_int), ("us", C.c_double), ("candidates", C.c_int)]


BATCH_MIXED = 0
BATCH_FP64 = 1


class TuneResult(C.Structure):
    _fields_ = [("kernel", C.c_int), ("width", C.c_int), ("block", C.c_int),
                ("us", C.c_double), ("candidates", C.c_int)]


_p = C.c_void_p
_i32 = C.c_int32
_i64 = C.c_int64
_int = C.c_int
_pp = C.POINTER(C.c_void_p)

# name: (argtypes) -- every function returns int status.
_SIGS = {
    "spmv_get_version": [C.POINTER(_int), C.POINTER(_int)],
    "spmv_comm_create": [_int, _p, _int, C.POINTER(_p)],
    "spmv_comm_destroy": [_p],
    "spmv_comm_size": [_p, C.POINTER(_int)],
    "spmv_comm_device": [_p, C.POINTER(_int)],
    "spmv_comm_stream": [_p, C.POINTER(_p)],
    "spmv_comm_synchronize": [_p],
    "spmv_l2gmap_create": [_p, C.POINTER(_i64), C.POINTER(C.POINTER(_i64)),
                           C.POINTER(_i64), C.POINTER(_p)],
    "spmv_l2gmap_destroy": [_p],
    "spmv_l2gmap_local_size": [_p, _int, C.POINTER(_i32)],
    "spmv_l2gmap_num_ghosts": [_p, _int, C.POINTER(_i32)],
    "spmv_l2gmap_global_size": [_p, C.POINTER(_i64)],
    "spmv_l2gmap_global_offset": [_p, _int, C.POINTER(_i64)],
    "spmv_l2gmap_global_to_local": [_p, _int, _i64, C.POINTER(_i32)],
    "spmv_l2gmap_ghosts": [_p, _int, C.POINTER(C.POINTER(_i64)), C.POINTER(_i32)],
    "spmv_l2gmap_pattern": [_p, _int, _int, C.POINTER(C.POINTER(_i32)),
                            C.POINTER(_i32)],
    "spmv_l2gmap_update": [_p, _int, _int, _pp],
    "spmv_l2gmap_reverse_update": [_p, _int, _int, _pp],
    "spmv_matrix_create_csr": [_p, _int, _p, _p, C.POINTER(_i32), C.POINTER(_i32),
                               _pp, _pp, _pp, C.POINTER(_p)],
    "spmv_matrix_destroy": [_p],
    "spmv_matrix_mult": [_p, _int, _pp, _pp],
    "spmv_matrix_transpmult": [_p, _int, _pp, _pp],
    "spmv_matrix_dtype": [_p, C.POINTER(_int)],
    "spmv_matrix_rows": [_p, _int, C.POINTER(_i32)],
    "spmv_matrix_cols": [_p, _int, C.POINTER(_i32)],
    "spmv_matrix_nnz": [_p, _int, C.POINTER(_i64)],
    "spmv_matrix_csr": [_p, _int, C.POINTER(C.POINTER(_i32)),
                        C.POINTER(C.POINTER(_i32)), C.POINTER(_p)],
    "spmv_matrix_col_map": [_p, C.POINTER(_p)],
    "spmv_matrix_row_map": [_p, C.POINTER(_p)],
    "spmv_matrix_set_values": [_p, _int, _pp],
    "spmv_matrix_mult_noalloc": [_p, _pp, _pp],
    "spmv_matrix_set_kernel": [_p, _int, _int, _int],
    "spmv_matrix_get_kernel": [_p, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int)],
    "spmv_cg": [_p, _int, _pp, C.POINTER(_i64), _pp, _int, C.c_double,
                C.POINTER(_int)],
    "spmv_cg_ex": [_p, _int, _pp, C.POINTER(_i64), _pp, _int, C.c_double,
                   C.POINTER(CgInfo)],
    "spmv_cg_mixed": [_p, _int, _pp, C.POINTER(_i64), _pp, _int, C.c_double,
                      C.POINTER(IrInfo)],
    "spmv_matrix_sample_outer": [_p, _int, C.c_double, _pp, _pp, _pp],
    "spmv_batch_create": [_p, _int, C.POINTER(_i32), _pp, _pp, _pp, C.POINTER(_p)],
    "spmv_batch_destroy": [_p],
    "spmv_batch_set_block": [_p, _int, _int],
    "spmv_batch_set_config": [_p, _int, C.POINTER(BatchConfig)],
    "spmv_batch_get_config": [_p, _int, C.POINTER(BatchConfig)],
    "spmv_batch_autotune": [_p, _int, C.POINTER(BatchConfig)],
    "spmv_batch_stats": [_p, C.POINTER(_i64), C.POINTER(_i64), C.POINTER(_i64),
                         C.POINTER(_int)],
    "spmv_batch_solve_ex": [_p, _int, _int, _pp, _pp, _p, _p, _int, C.c_double,
                            C.POINTER(IrInfo), C.POINTER(IrInfo)],
    "spmv_batch_solve": [_p, _int, _pp, _pp, _int, C.c_double, C.POINTER(IrInfo)],
    "spmv_matrix_autotune": [_p, _int, C.POINTER(TuneResult)],
    "spmv_matrix_cg_form": [_p, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int)],
    "spmv_matrix_cg_mixed_form": [_p, C.POINTER(_int), C.POINTER(_int), C.POINTER(_int)],
    "spmv_matrix_solver_product": [_p, _int, C.POINTER(_int), C.POINTER(_int),
                                   C.POINTER(_int), C.POINTER(C.c_double)],
    "spmv_matrix_mult_block": [_p, _int, _int, _pp, _pp],
    "spmv_cg_block": [_p, _int, _int, _pp, _pp, _int, C.c_double, C.POINTER(CgInfo)],
    "spmv_owner_ranges": [_int, _i64, C.POINTER(_i64)],
    "spmv_matrix_create_assembled": [_p, _int, C.POINTER(_i64), C.POINTER(_i64), _pp, _pp, _pp,
                                     _pp, C.POINTER(_i64), _pp, C.POINTER(_i64), C.POINTER(_p),
                                     C.POINTER(_p), C.POINTER(_p)],
    "spmv_petsc_read_matrix": [_p, C.c_char_p, C.POINTER(_p), C.POINTER(_p), C.POINTER(_p)],
    "spmv_petsc_vector_size": [C.c_char_p, C.POINTER(_i64)],
    "spmv_petsc_read_vector": [_p, C.c_char_p, _pp],
}

_lib = None


def lib():
    """Loads libspmv_b200.so (once).  Raises if it has not been built: there
    is no fallback path."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m spmv_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, args in _SIGS.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.spmv_last_error.argtypes = []
        L.spmv_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != SUCCESS:
        msg = lib().spmv_last_error().decode("utf-8", "replace")
        raise SpmvError(status, msg)


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args))


def ptr_array(ptrs) -> "C.Array":
    """void*[n] from a sequence of integer addresses (or None)."""
    arr = (C.c_void_p * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


def declared_symbols(header: Path | None = None):
    """Names of the functions declared in include/spmv_b200.h."""
    import re
    header = header or (PKG.parent / "include" / "spmv_b200.h")
    text = header.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\**(spmv_\w+)\s*\(",
                                 text, flags=re.M)))

