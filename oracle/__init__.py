"""ORACLE - TEST INFRASTRUCTURE ONLY.

Python access to the CPU restatement of libspmv's hot path (oracle.cpp),
plus the recipe that builds it.  Only the tests, the smoke check and the
CPU-baseline leg of bench.py may use this package; the product never does.
Parity is unpinned: the reference cannot be built here and ships no golden
outputs (see oracle.cpp's header).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import List, Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_spmv.so"
_lib = None


def build(force: bool = False) -> Path:
    src = HERE / "oracle.cpp"
    if force or not LIB_PATH.exists() or src.stat().st_mtime > LIB_PATH.stat().st_mtime:
        subprocess.run(["make", "-C", str(HERE), "-B" if force else "-s"], check=True,
                       capture_output=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: run `make -C oracle`")
        L = C.CDLL(str(LIB_PATH))
        P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_owner_ranges.argtypes = [I64, I64, P]
        L.oracle_map_create.argtypes = [C.c_int, P, P, P, C.POINTER(P)]
        L.oracle_map_free.argtypes = [P]
        L.oracle_map_field.argtypes = [P, C.c_int, C.c_int,
                                       C.POINTER(C.POINTER(I32)), C.POINTER(I32)]
        L.oracle_map_global_to_local.argtypes = [P, C.c_int, I64]
        L.oracle_map_global_to_local.restype = I32
        for n in ("oracle_update_f64", "oracle_update_f32", "oracle_reverse_update_f64",
                  "oracle_reverse_update_f32"):
            getattr(L, n).argtypes = [P, P]
        L.oracle_csr_mult_f64.argtypes = [I32, P, P, P, P, P, C.c_int]
        L.oracle_csr_mult_f32.argtypes = [I32, P, P, P, P, P]
        L.oracle_csr_transpmult_f64.argtypes = [I32, I32, P, P, P, P, P]
        L.oracle_csr_transpmult_f32.argtypes = [I32, I32, P, P, P, P, P]
        for n in ("oracle_csr_mult_c128", "oracle_csr_mult_c64"):
            getattr(L, n).argtypes = [I32, P, P, P, P, P]
        for n in ("oracle_csr_transpmult_c128", "oracle_csr_transpmult_c64"):
            getattr(L, n).argtypes = [I32, I32, P, P, P, P, P]
        L.oracle_cg.argtypes = [P, C.c_int, P, P, P, P, P, P, C.c_int, D, C.c_int,
                                C.c_int, C.POINTER(D)]
        L.oracle_cg.restype = C.c_int
        L.oracle_matvec_demo.argtypes = [C.c_int, I64, C.c_int]
        L.oracle_matvec_demo.restype = D
        L.oracle_max_threads.restype = C.c_int
        L.oracle_petsc_read.argtypes = [C.c_char_p, C.c_int]
        L.oracle_petsc_read.restype = P
        L.oracle_petsc_free.argtypes = [P]
        L.oracle_petsc_block.argtypes = [P, C.c_int, C.c_int, C.POINTER(P)]
        L.oracle_petsc_block.restype = I64
        L.oracle_create_matrix.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P]
        L.oracle_create_matrix.restype = P
        L.oracle_assembled_free.argtypes = [P]
        L.oracle_assembled_block.argtypes = [P, C.c_int, C.c_int, C.POINTER(P)]
        L.oracle_assembled_block.restype = I64
        _lib = L
    return _lib


def _parr(arrs):
    out = (C.c_void_p * max(1, len(arrs)))()
    for i, a in enumerate(arrs):
        out[i] = a.ctypes.data
    return out


def owner_ranges(size: int, N: int) -> np.ndarray:
    out = np.zeros(size + 1, np.int64)
    lib().oracle_owner_ranges(size, N, out.ctypes.data)
    return out


class Map:
    """The reference's L2GMap for all ranks (L2GMap.cpp:15-122 restated)."""

    def __init__(self, local_sizes: Sequence[int], ghosts: Sequence[np.ndarray]):
        self.P = len(local_sizes)
        self._ls = np.asarray(local_sizes, np.int64)
        self._g = [np.ascontiguousarray(g, np.int64) for g in ghosts]
        self._ng = np.array([len(g) for g in self._g], np.int64)
        h = C.c_void_p()
        if lib().oracle_map_create(self.P, self._ls.ctypes.data, _parr(self._g),
                                   self._ng.ctypes.data, C.byref(h)) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        self._h = h

    def field(self, rank: int, name: str) -> np.ndarray:
        idx = {"neighbours": 0, "send_count": 1, "recv_count": 2, "send_offset": 3,
               "recv_offset": 4, "indexbuf": 5}[name]
        p, n = C.POINTER(C.c_int32)(), C.c_int32()
        if lib().oracle_map_field(self._h, rank, idx, C.byref(p), C.byref(n)) != 0:
            raise RuntimeError(lib().oracle_last_error().decode())
        return np.ctypeslib.as_array(p, (n.value,)).copy() if n.value else \
            np.zeros(0, np.int32)

    def global_to_local(self, rank: int, i: int) -> int:
        return lib().oracle_map_global_to_local(self._h, rank, i)

    def update(self, vecs: List[np.ndarray]) -> None:
        f = lib().oracle_update_f64 if vecs[0].dtype == np.float64 else lib().oracle_update_f32
        f(self._h, _parr(vecs))

    def reverse_update(self, vecs: List[np.ndarray]) -> None:
        f = (lib().oracle_reverse_update_f64 if vecs[0].dtype == np.float64
             else lib().oracle_reverse_update_f32)
        f(self._h, _parr(vecs))

    def __del__(self):
        try:
            lib().oracle_map_free(self._h)
        except Exception:
            pass


def csr_mult(rp, ci, v, x, nthreads: int = 1) -> np.ndarray:
    """Matrix::operator* restated (Eigen's row loop, storage order)."""
    m = len(rp) - 1
    rp = np.ascontiguousarray(rp, np.int32)
    ci = np.ascontiguousarray(ci, np.int32)
    v = np.ascontiguousarray(v)
    x = np.ascontiguousarray(x, v.dtype)
    y = np.empty(m, v.dtype)
    args = (m, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, x.ctypes.data, y.ctypes.data)
    if v.dtype == np.float64:
        lib().oracle_csr_mult_f64(*args, nthreads)
    elif v.dtype == np.float32:
        lib().oracle_csr_mult_f32(*args)
    elif v.dtype == np.complex128:
        lib().oracle_csr_mult_c128(*args)
    elif v.dtype == np.complex64:
        lib().oracle_csr_mult_c64(*args)
    else:
        raise TypeError(v.dtype)
    return y


def csr_transpmult(rp, ci, v, x, ncols: int) -> np.ndarray:
    """Matrix::transpmult restated (column scatter, no conjugation)."""
    m = len(rp) - 1
    rp = np.ascontiguousarray(rp, np.int32)
    ci = np.ascontiguousarray(ci, np.int32)
    v = np.ascontiguousarray(v)
    x = np.ascontiguousarray(x, v.dtype)
    y = np.empty(ncols, v.dtype)
    f = {np.dtype(np.float64): lib().oracle_csr_transpmult_f64,
         np.dtype(np.float32): lib().oracle_csr_transpmult_f32,
         np.dtype(np.complex128): lib().oracle_csr_transpmult_c128,
         np.dtype(np.complex64): lib().oracle_csr_transpmult_c64}[v.dtype]
    f(m, ncols, rp.ctypes.data, ci.ctypes.data, v.ctypes.data, x.ctypes.data,
      y.ctypes.data)
    return y


def cg(col_map: Map, blocks, b: List[np.ndarray], max_its: int, rtol: float,
       nthreads: int = 1, max_its_run: int | None = None):
    """spmv::cg (cg.cpp:11-83) restated; returns (x per rank, k, rnorm)."""
    P = col_map.P
    nrows = np.array([len(blk[0]) - 1 for blk in blocks], np.int32)
    rps = [np.ascontiguousarray(blk[0], np.int32) for blk in blocks]
    cis = [np.ascontiguousarray(blk[1], np.int32) for blk in blocks]
    vas = [np.ascontiguousarray(blk[2], np.float64) for blk in blocks]
    bs = [np.ascontiguousarray(v, np.float64) for v in b]
    xs = [np.zeros(col_map._ls[q] + col_map._ng[q]) for q in range(P)]
    rn = C.c_double()
    k = lib().oracle_cg(col_map._h, P, nrows.ctypes.data, _parr(rps), _parr(cis),
                        _parr(vas), _parr(bs), _parr(xs), max_its, rtol, nthreads,
                        max_its if max_its_run is None else max_its_run, C.byref(rn))
    return xs, k, rn.value


def matvec_demo(P: int, N: int = 500000, n_apply: int = 1000) -> float:
    return lib().oracle_matvec_demo(P, N, n_apply)


def max_threads() -> int:
    return lib().oracle_max_threads()


def petsc_read(filename, P: int):
    """read_petsc_binary restated (read_petsc.cpp:32-191) for P ranks:
    per rank [rowptr, colind, values, ghosts]."""
    L = lib()
    h = L.oracle_petsc_read(str(filename).encode(), int(P))
    if not h:
        raise RuntimeError(L.oracle_last_error().decode())
    try:
        out = []
        for r in range(P):
            arrs = []
            for field, ct, dt in ((0, C.c_int32, np.int32), (1, C.c_int32, np.int32),
                                  (2, C.c_double, np.float64), (3, C.c_int64, np.int64)):
                p = C.c_void_p()
                n = L.oracle_petsc_block(h, r, field, C.byref(p))
                arrs.append(np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), (n,)).copy()
                            if n > 0 else np.zeros(0, dt))
            out.append(arrs)
        return out
    finally:
        L.oracle_petsc_free(h)


def create_matrix(blocks, nrows_local, ncols_local, row_ghosts, col_ghosts):
    """Matrix::create_matrix restated (Matrix.cpp:213-438): per rank
    [rowptr, colind, values, ghosts] of the assembled matrix (values in the
    blocks' dtype: float64 or complex128)."""
    L = lib()
    P = len(blocks)
    cplx = np.iscomplexobj(blocks[0][2])
    keep = []

    def arr(a, dt):
        a = np.ascontiguousarray(a, dt)
        keep.append(a)
        return a.ctypes.data if len(a) else None

    def parr(addrs):
        out = (C.c_void_p * max(1, len(addrs)))()
        for i, a in enumerate(addrs):
            out[i] = a
        return out

    rp = parr([arr(b[0], np.int32) for b in blocks])
    ci = parr([arr(b[1], np.int32) for b in blocks])
    va = parr([arr(b[2], np.complex128 if cplx else np.float64) for b in blocks])
    rg = parr([arr(g, np.int64) for g in row_ghosts])
    cg_ = parr([arr(g, np.int64) for g in col_ghosts])
    i64 = lambda v: (C.c_int64 * P)(*[int(t) for t in v])  # noqa: E731
    h = L.oracle_create_matrix(P, 1 if cplx else 0, i64(nrows_local), i64(ncols_local), rp, ci,
                               va, rg, i64([len(g) for g in row_ghosts]), cg_,
                               i64([len(g) for g in col_ghosts]))
    if not h:
        raise RuntimeError(L.oracle_last_error().decode())
    try:
        out = []
        for r in range(P):
            arrs = []
            for field, ct, dt in ((0, C.c_int32, np.int32), (1, C.c_int32, np.int32),
                                  (2, C.c_double, np.float64), (3, C.c_int64, np.int64)):
                p = C.c_void_p()
                n = L.oracle_assembled_block(h, r, field, C.byref(p))
                m = 2 * n if field == 2 else n
                a = (np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), (m,)).copy()
                     if n > 0 else np.zeros(m, dt))
                if field == 2:
                    a = a.view(np.complex128)
                    if not cplx:
                        a = a.real.copy()
                arrs.append(a)
            out.append(arrs)
        return out
    finally:
        L.oracle_assembled_free(h)
