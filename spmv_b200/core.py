"""Python mirror of libspmv's hot-path API over the C ABI.

Names and argument meanings follow the reference (spmv::L2GMap, spmv::Matrix,
spmv::cg); because the ranks of the reference's MPI communicator are virtual
ranks on one GPU here, the collective calls take one entry per rank in lists.

Vectors are numpy arrays (host memory: the call copies to the device and
back) or CUDA torch tensors (device memory: used in place, ordered on the
communicator's stream).  Errors raise SpmvError (a RuntimeError) carrying the
reference's message where it has one.
"""
from __future__ import annotations

import ctypes as C
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import SpmvError, call, ptr_array

_DTYPES = {np.dtype(np.float64): _lib.FLOAT64, np.dtype(np.float32): _lib.FLOAT32,
           np.dtype(np.complex64): _lib.COMPLEX64,
           np.dtype(np.complex128): _lib.COMPLEX128}
_NP_OF = {v: k for k, v in _DTYPES.items()}


def _is_torch(v) -> bool:
    return type(v).__module__.startswith("torch")


class _Fence:
    """Orders library work after and before torch work on device tensors.

    The communicator's CUDA stream is not torch's current stream, so on entry
    the library stream waits for work already queued on torch's stream (that
    produced the inputs), and on exit torch's stream waits for the library's
    work (that produces the outputs).  Both waits are device-side events; the
    host does not block."""

    def __init__(self, comm, device: bool):
        self.comm = comm if device else None

    def __enter__(self):
        if self.comm is not None:
            import torch
            self.torch_stream = torch.cuda.current_stream(self.comm.device)
            self.lib_stream = self.comm.torch_stream()
            self.lib_stream.wait_stream(self.torch_stream)
        return self

    def __exit__(self, *exc):
        if self.comm is not None:
            self.torch_stream.wait_stream(self.lib_stream)
        return False


def _vec_info(vecs: Sequence):
    """(memory kind, dtype code, addresses) of a per-rank vector list."""
    if len(vecs) == 0:
        raise SpmvError(_lib.ERROR_INVALID_ARGUMENT, "spmv: empty vector list")
    kinds = {_is_torch(v) for v in vecs}
    if len(kinds) != 1:
        raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                        "spmv: mix of host and device vectors")
    if kinds.pop():
        import torch
        for v in vecs:
            if not v.is_cuda or not v.is_contiguous():
                raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                                "spmv: device vectors must be contiguous CUDA tensors")
        tdt = {torch.float64: _lib.FLOAT64, torch.float32: _lib.FLOAT32,
               torch.complex64: _lib.COMPLEX64, torch.complex128: _lib.COMPLEX128}
        dts = {tdt.get(v.dtype, -1) for v in vecs}
        ptrs = [v.data_ptr() for v in vecs]
        mem = _lib.MEMORY_DEVICE
    else:
        for v in vecs:
            if not (isinstance(v, np.ndarray) and v.flags.c_contiguous):
                raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                                "spmv: host vectors must be contiguous numpy arrays")
        dts = {_DTYPES.get(v.dtype, -1) for v in vecs}
        ptrs = [v.ctypes.data for v in vecs]
        mem = _lib.MEMORY_HOST
    if len(dts) != 1 or -1 in dts:
        raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                        "spmv: vectors need one supported dtype")
    return mem, dts.pop(), ptrs


class Comm:
    """Virtual communicator: `size` ranks on CUDA device `device` (-1 for a
    host-only communicator that can build and inspect maps and matrices).
    `stream` is a cudaStream_t handle (int) or None for a library stream."""

    def __init__(self, size: int = 1, device: int = 0, stream: Optional[int] = None):
        h = C.c_void_p()
        call("spmv_comm_create", device, stream, size, C.byref(h))
        self._h = h
        self.size = size
        self.device = device

    @property
    def handle(self):
        return self._h

    @property
    def stream(self) -> int:
        s = C.c_void_p()
        call("spmv_comm_stream", self._h, C.byref(s))
        return s.value or 0

    def synchronize(self) -> None:
        call("spmv_comm_synchronize", self._h)

    def torch_stream(self):
        """The communicator's stream as a torch.cuda.ExternalStream."""
        if getattr(self, "_ts", None) is None:
            import torch
            self._ts = torch.cuda.ExternalStream(self.stream,
                                                 device=torch.device("cuda", self.device))
        return self._ts

    def fence(self, vecs) -> "_Fence":
        return _Fence(self, bool(vecs) and _is_torch(vecs[0]))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().spmv_comm_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class L2GMap:
    """spmv::L2GMap (L2GMap.h:14-97) for every rank of `comm` at once:
    local_sizes[r] owned entries and sorted ghost global indices ghosts[r]."""

    def __init__(self, comm: Comm, local_sizes: Sequence[int],
                 ghosts: Sequence[Sequence[int]]):
        P = comm.size
        if len(local_sizes) != P or len(ghosts) != P:
            raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                            "spmv::L2GMap - Error: need one entry per rank")
        self.comm = comm
        ls = (C.c_int64 * P)(*[int(v) for v in local_sizes])
        self._g = [np.ascontiguousarray(np.asarray(g, dtype=np.int64)) for g in ghosts]
        gp = (C.POINTER(C.c_int64) * P)(
            *[g.ctypes.data_as(C.POINTER(C.c_int64)) for g in self._g])
        ng = (C.c_int64 * P)(*[len(g) for g in self._g])
        h = C.c_void_p()
        call("spmv_l2gmap_create", comm.handle, ls, gp, ng, C.byref(h))
        self._h = h

    @property
    def handle(self):
        return self._h

    def local_size(self, rank: int) -> int:
        v = C.c_int32()
        call("spmv_l2gmap_local_size", self._h, rank, C.byref(v))
        return v.value

    def num_ghosts(self, rank: int) -> int:
        v = C.c_int32()
        call("spmv_l2gmap_num_ghosts", self._h, rank, C.byref(v))
        return v.value

    def global_size(self) -> int:
        v = C.c_int64()
        call("spmv_l2gmap_global_size", self._h, C.byref(v))
        return v.value

    def global_offset(self, rank: int) -> int:
        v = C.c_int64()
        call("spmv_l2gmap_global_offset", self._h, rank, C.byref(v))
        return v.value

    def global_to_local(self, rank: int, i: int) -> int:
        v = C.c_int32()
        call("spmv_l2gmap_global_to_local", self._h, rank, int(i), C.byref(v))
        return v.value

    def ghosts(self, rank: int) -> np.ndarray:
        p = C.POINTER(C.c_int64)()
        n = C.c_int32()
        call("spmv_l2gmap_ghosts", self._h, rank, C.byref(p), C.byref(n))
        return np.ctypeslib.as_array(p, (n.value,)).copy() if n.value else \
            np.zeros(0, np.int64)

    def pattern(self, rank: int, field: str) -> np.ndarray:
        p = C.POINTER(C.c_int32)()
        n = C.c_int32()
        call("spmv_l2gmap_pattern", self._h, rank, _lib.PATTERN_FIELDS[field],
             C.byref(p), C.byref(n))
        return np.ctypeslib.as_array(p, (n.value,)).copy() if n.value else \
            np.zeros(0, np.int32)

    def vec_len(self, rank: int) -> int:
        return self.local_size(rank) + self.num_ghosts(rank)

    def update(self, vecs: Sequence) -> None:
        """L2GMap::update (L2GMap.cpp:126-150) on all ranks' vectors, in place."""
        mem, dt, ptrs = _vec_info(vecs)
        with self.comm.fence(vecs):
            call("spmv_l2gmap_update", self._h, dt, mem, ptr_array(ptrs))

    def reverse_update(self, vecs: Sequence) -> None:
        """L2GMap::reverse_update (L2GMap.cpp:152-170), in place."""
        mem, dt, ptrs = _vec_info(vecs)
        with self.comm.fence(vecs):
            call("spmv_l2gmap_reverse_update", self._h, dt, mem, ptr_array(ptrs))

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().spmv_l2gmap_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Matrix:
    """spmv::Matrix<T> (Matrix.h:23-81): rank r's local CSR block
    blocks[r] = (rowptr, colind, values) with columns numbered owned-then-
    ghosts by col_map.  The block is copied in, as the reference's
    constructor copies its Eigen matrix."""

    def __init__(self, comm: Comm, blocks, col_map: Optional[L2GMap],
                 row_map: Optional[L2GMap], nrows=None, ncols=None):
        P = comm.size
        if len(blocks) != P:
            raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                            "spmv::Matrix - Error: need one block per rank")
        self.comm, self._col_map, self._row_map = comm, col_map, row_map
        rps, cis, vas = [], [], []
        for (rp, ci, va) in blocks:
            rps.append(np.ascontiguousarray(rp, dtype=np.int32))
            cis.append(np.ascontiguousarray(ci, dtype=np.int32))
            vas.append(np.ascontiguousarray(va))
        dts = {v.dtype for v in vas}
        if len(dts) != 1 or next(iter(dts)) not in _DTYPES:
            raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                            "spmv::Matrix - Error: values need one supported dtype")
        self.np_dtype = next(iter(dts))
        self.dtype = _DTYPES[self.np_dtype]
        if nrows is None:
            nrows = [len(rp) - 1 for rp in rps]
        if ncols is None:
            if col_map is None:
                raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                                "spmv::Matrix - Error: ncols needed without col_map")
            ncols = [col_map.vec_len(r) for r in range(P)]
        nr = (C.c_int32 * P)(*nrows)
        nc = (C.c_int32 * P)(*ncols)
        h = C.c_void_p()
        call("spmv_matrix_create_csr", comm.handle, self.dtype,
             col_map.handle if col_map else None, row_map.handle if row_map else None,
             nr, nc, ptr_array([a.ctypes.data for a in rps]),
             ptr_array([a.ctypes.data for a in cis]),
             ptr_array([a.ctypes.data for a in vas]), C.byref(h))
        self._h = h
        self.nrows = list(nrows)
        self.ncols = list(ncols)

    @property
    def handle(self):
        return self._h

    def row_map(self) -> Optional[L2GMap]:
        return self._row_map

    def col_map(self) -> Optional[L2GMap]:
        return self._col_map

    def nnz(self, rank: int) -> int:
        v = C.c_int64()
        call("spmv_matrix_nnz", self._h, rank, C.byref(v))
        return v.value

    def mat(self, rank: int):
        """Matrix::mat(): copies of rank's host CSR arrays."""
        rp, ci, va = C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(), C.c_void_p()
        call("spmv_matrix_csr", self._h, rank, C.byref(rp), C.byref(ci), C.byref(va))
        m, nnz = self.nrows[rank], self.nnz(rank)
        rpa = np.ctypeslib.as_array(rp, (m + 1,)).copy()
        cia = np.ctypeslib.as_array(ci, (nnz,)).copy() if nnz else np.zeros(0, np.int32)
        buf = (C.c_char * (nnz * self.np_dtype.itemsize)).from_address(va.value) \
            if nnz else b""
        vaa = np.frombuffer(bytes(buf), dtype=self.np_dtype).copy()
        return rpa, cia, vaa

    def set_values(self, values: Sequence) -> None:
        mem, dt, ptrs = _vec_info(values)
        with self.comm.fence(values):
            call("spmv_matrix_set_values", self._h, mem, ptr_array(ptrs))

    def set_kernel(self, kernel: str = "auto", width: int = 0, block: int = 0) -> None:
        k = {"auto": _lib.KERNEL_AUTO, "vector": _lib.KERNEL_VECTOR,
             "merge": _lib.KERNEL_MERGE, "sell": _lib.KERNEL_SELL,
             "staged": _lib.KERNEL_STAGED}[kernel]
        call("spmv_matrix_set_kernel", self._h, k, width, block)

    def mult_block(self, X: Sequence, out: Optional[List] = None) -> List:
        """Y[r] = A[r] X[r] for X[r] of shape (ncols[r], k), k <= 32, row-major."""
        mem, dt, ptrs = _vec_info(X)
        k = int(X[0].shape[1])
        if out is None:
            if _is_torch(X[0]):
                import torch
                out = [torch.empty((n, k), dtype=X[0].dtype, device=X[0].device)
                       for n in self.nrows]
            else:
                out = [np.empty((n, k), dtype=X[0].dtype) for n in self.nrows]
        _, _, optrs = _vec_info(out)
        with self.comm.fence(X):
            call("spmv_matrix_mult_block", self._h, k, mem, ptr_array(ptrs),
                 ptr_array(optrs))
        return out

    def autotune(self, reps: int = 10):
        """Times the candidate kernels on this matrix and keeps the fastest;
        returns (kernel, width, block, microseconds, candidates timed)."""
        r = _lib.TuneResult()
        call("spmv_matrix_autotune", self._h, int(reps), C.byref(r))
        names = _lib.KERNEL_NAMES
        return names[r.kernel], r.width, r.block, r.us, r.candidates

    def solver_product(self, solver: str = "cg"):
        """The product a solver of this matrix runs: solver "cg", "mixed32"
        (FP32 inner product of cg_mixed) or "mixed64" (its FP64 residual).
        Returns (kernel, width, index_bits, microseconds of the plain
        product); fails if that solver has not run on the matrix."""
        s = {"cg": 0, "mixed32": 1, "mixed64": 2}[solver]
        k, w, bits, us = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        call("spmv_matrix_solver_product", self._h, s, C.byref(k), C.byref(w),
             C.byref(bits), C.byref(us))
        return _lib.KERNEL_NAMES[k.value], w.value, bits.value, us.value

    def cg_form(self, solver="cg"):
        """How cg (solver="cg") or cg_mixed (solver="mixed") runs on this
        matrix: ("graph", 0, None) for its kernels in a CUDA graph, or
        ("fused", CTAs per SM, "smem" or "global": where the residual lives)
        for one cooperative launch per solve, with ":m" appended for cg's
        merged-update form (two grid syncs per iteration); fails if that
        solver has not run on the matrix."""
        fn = {"cg": "spmv_matrix_cg_form", "mixed": "spmv_matrix_cg_mixed_form"}[solver]
        f, cps, rs = C.c_int(), C.c_int(), C.c_int()
        call(fn, self._h, C.byref(f), C.byref(cps), C.byref(rs))
        if not f.value:
            return "graph", 0, None
        where = "smem" if rs.value else "global"
        return "fused", cps.value, where + (":m" if f.value == 2 else "")

    def get_kernel(self):
        k, w, b = C.c_int(), C.c_int(), C.c_int()
        call("spmv_matrix_get_kernel", self._h, C.byref(k), C.byref(w), C.byref(b))
        return _lib.KERNEL_NAMES[k.value], w.value, b.value

    def _alloc_like(self, x0, lens):
        if _is_torch(x0):
            import torch
            return [torch.empty(n, dtype=x0.dtype, device=x0.device) for n in lens]
        return [np.empty(n, dtype=x0.dtype) for n in lens]

    def mult(self, x: Sequence, out: Optional[List] = None) -> List:
        """Matrix::operator* (Matrix.cpp:158-166): y[r] = A[r] x[r]."""
        mem, dt, ptrs = _vec_info(x)
        y = out if out is not None else self._alloc_like(x[0], self.nrows)
        _, _, yptrs = _vec_info(y)
        with self.comm.fence(x):
            call("spmv_matrix_mult", self._h, mem, ptr_array(ptrs), ptr_array(yptrs))
        return y

    __mul__ = mult

    def transpmult(self, x: Sequence, out: Optional[List] = None) -> List:
        """Matrix::transpmult (Matrix.cpp:168-176): y[r] = A[r]^T x[r]."""
        mem, dt, ptrs = _vec_info(x)
        y = out if out is not None else self._alloc_like(x[0], self.ncols)
        _, _, yptrs = _vec_info(y)
        with self.comm.fence(x):
            call("spmv_matrix_transpmult", self._h, mem, ptr_array(ptrs),
                 ptr_array(yptrs))
        return y

    def sample_outer(self, lam: Sequence, x: Sequence, scale: float = -1.0,
                     out: Optional[List] = None) -> List:
        """out[r][k] = scale * lam[r][row(k)] * x[r][col(k)] on every stored
        entry (dL/dA on A's pattern for scale = -1, lam the adjoint)."""
        mem, dt, lptrs = _vec_info(lam)
        _, _, xptrs = _vec_info(x)
        if out is None:
            out = self._alloc_like(lam[0], [self.nnz(r) for r in range(self.comm.size)])
        _, _, optrs = _vec_info(out)
        with self.comm.fence(lam):
            call("spmv_matrix_sample_outer", self._h, mem, float(scale),
                 ptr_array(lptrs), ptr_array(xptrs), ptr_array(optrs))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().spmv_matrix_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def cg(comm: Comm, A: Matrix, b: Sequence, max_its: int, rtol: float,
       x: Optional[List] = None, info: bool = False):
    """spmv::cg (cg.cpp:11-83) on all ranks: returns (x, k), x[r] of length
    col_map local_size + num_ghosts (ghost tail zero).  With info=True returns
    (x, k, CgInfo)."""
    if comm is not A.comm:
        raise SpmvError(_lib.ERROR_INVALID_ARGUMENT, "spmv::cg - Error: comm mismatch")
    mem, dt, bptrs = _vec_info(b)
    cm = A.col_map()
    if x is None:
        lens = [cm.vec_len(r) for r in range(comm.size)] if cm else A.ncols
        x = A._alloc_like(b[0], lens)
    _, _, xptrs = _vec_info(x)
    rows = (C.c_int64 * comm.size)(*[len(v) for v in b])
    ci = _lib.CgInfo()
    with comm.fence(b):
        st = _lib.lib().spmv_cg_ex(A.handle, mem, ptr_array(bptrs), rows,
                                   ptr_array(xptrs), int(max_its), float(rtol),
                                   C.byref(ci))
    _lib.check(st)
    if info:
        return x, ci.iterations, ci
    return x, ci.iterations


def cg_mixed(comm: Comm, A: Matrix, b: Sequence, max_its: int, rtol: float,
             x: Optional[List] = None):
    """Mixed-precision CG (FP32 inner iterations, FP64 refinement) to
    ||b - A x|| / ||b|| < rtol confirmed in FP64.  Returns (x, IrInfo)."""
    if comm is not A.comm:
        raise SpmvError(_lib.ERROR_INVALID_ARGUMENT, "spmv::cg - Error: comm mismatch")
    mem, dt, bptrs = _vec_info(b)
    cm = A.col_map()
    if x is None:
        x = A._alloc_like(b[0], [cm.vec_len(r) for r in range(comm.size)])
    _, _, xptrs = _vec_info(x)
    rows = (C.c_int64 * comm.size)(*[len(v) for v in b])
    info = _lib.IrInfo()
    with comm.fence(b):
        st = _lib.lib().spmv_cg_mixed(A.handle, mem, ptr_array(bptrs), rows,
                                      ptr_array(xptrs), int(max_its), float(rtol),
                                      C.byref(info))
    _lib.check(st)
    return x, info


def cg_block(comm: Comm, A: Matrix, B: Sequence, max_its: int, rtol: float,
             X: Optional[List] = None):
    """Block CG: k independent solves (B[r] of shape (local_size, k)) sharing
    one SpMM per iteration.  Returns (X, [CgInfo] * k)."""
    mem, dt, bptrs = _vec_info(B)
    k = int(B[0].shape[1])
    cm = A.col_map()
    if X is None:
        lens = [cm.vec_len(r) for r in range(comm.size)]
        if _is_torch(B[0]):
            import torch
            X = [torch.empty((n, k), dtype=B[0].dtype, device=B[0].device) for n in lens]
        else:
            X = [np.empty((n, k), dtype=B[0].dtype) for n in lens]
    _, _, xptrs = _vec_info(X)
    info = (_lib.CgInfo * k)()
    with comm.fence(B):
        call("spmv_cg_block", A.handle, k, mem, ptr_array(bptrs), ptr_array(xptrs),
             int(max_its), float(rtol), info)
    return X, list(info)


class Batch:
    """Many independent SPD systems (one CSR each, symmetric pattern) solved
    together by spmv_batch_solve_ex: one cooperative launch in which every
    system's CG iterations run in lockstep, FP32 inner iterations with FP64
    refinement (or plain FP64).  `block=(system, nrhs)` adds a block of nrhs
    right-hand sides for one system, solved in the same launch with one
    product per iteration for all its columns."""

    def __init__(self, comm: Comm, systems, block: Optional[tuple] = None):
        self.comm = comm
        self._rp = [np.ascontiguousarray(s[0], np.int32) for s in systems]
        self._ci = [np.ascontiguousarray(s[1], np.int32) for s in systems]
        self._va = [np.ascontiguousarray(s[2], np.float64) for s in systems]
        self.n = [len(rp) - 1 for rp in self._rp]
        ns = len(systems)
        h = C.c_void_p()
        call("spmv_batch_create", comm.handle, ns, (C.c_int32 * max(ns, 1))(*self.n),
             ptr_array([a.ctypes.data for a in self._rp]),
             ptr_array([a.ctypes.data for a in self._ci]),
             ptr_array([a.ctypes.data for a in self._va]), C.byref(h))
        self._h = h
        # The library keeps its own (renumbered) copy.
        del self._rp, self._ci, self._va
        self.block = None
        if block is not None:
            self.set_block(*block)

    def set_block(self, system: int, nrhs: int) -> None:
        call("spmv_batch_set_block", self._h, int(system), int(nrhs))
        self.block = (int(system), int(nrhs))

    _PREC = {"mixed": _lib.BATCH_MIXED, "fp64": _lib.BATCH_FP64}

    def set_config(self, ctas_per_sm: int = 0, tile_rows: int = 0, rhs_lanes: int = 0,
                   window: Optional[bool] = None, precision: str = "mixed") -> None:
        w = 0 if window is None else (2 if window else 1)
        c = _lib.BatchConfig(int(ctas_per_sm), int(tile_rows), int(rhs_lanes), w, 0.0, 0)
        call("spmv_batch_set_config", self._h, self._PREC[precision], C.byref(c))

    @staticmethod
    def _cfg(c) -> dict:
        return {"ctas_per_sm": c.ctas_per_sm, "tile_rows": c.tile_rows,
                "rhs_lanes": c.rhs_lanes, "window": c.window == 2, "us": c.us,
                "candidates": c.candidates}

    def config(self, precision: str = "mixed") -> dict:
        c = _lib.BatchConfig()
        call("spmv_batch_get_config", self._h, self._PREC[precision], C.byref(c))
        return self._cfg(c)

    def autotune(self, precision: str = "mixed") -> dict:
        """Times the launch shapes on short solves of this precision and keeps
        the fastest for it."""
        c = _lib.BatchConfig()
        call("spmv_batch_autotune", self._h, self._PREC[precision], C.byref(c))
        return self._cfg(c)

    def stats(self) -> dict:
        rows, nnz, stored = C.c_int64(), C.c_int64(), C.c_int64()
        bits = C.c_int()
        call("spmv_batch_stats", self._h, C.byref(rows), C.byref(nnz), C.byref(stored),
             C.byref(bits))
        return {"rows": rows.value, "nnz": nnz.value, "stored": stored.value,
                "index_bits": bits.value}

    def solve(self, b: Sequence, max_its: int, rtol: float, x: Optional[List] = None,
              block_b=None, block_x=None, precision: str = "mixed"):
        """x[i] = A_i^-1 b[i] for every system (and X = A_s^-1 B for the block
        when block_b is given: n_s x nrhs, row-major).  Returns (x, info) or,
        with a block, (x, info, X, block_info)."""
        mem, dt, bptrs = _vec_info(b)
        if x is None:
            x = [np.empty_like(v) if not _is_torch(v) else v.new_empty(v.shape) for v in b]
        _, _, xptrs = _vec_info(x)
        info = (_lib.BatchInfo * max(len(b), 1))()
        binfo = None
        bb = bx = None
        if block_b is not None:
            if self.block is None:
                raise SpmvError(_lib.ERROR_INVALID_ARGUMENT, "spmv batch: no block was set")
            if block_x is None:
                block_x = (np.empty_like(block_b) if not _is_torch(block_b)
                           else block_b.new_empty(block_b.shape))
            bm, _, (bb,) = _vec_info([block_b])
            xm, _, (bx,) = _vec_info([block_x])
            if bm != mem or xm != mem:
                raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                                "spmv: mix of host and device vectors")
            binfo = (_lib.BatchInfo * self.block[1])()
        prec = self._PREC[precision]
        with self.comm.fence(b):
            call("spmv_batch_solve_ex", self._h, mem, prec, ptr_array(bptrs), ptr_array(xptrs),
                 bb, bx, int(max_its), float(rtol), info, binfo)
        if block_b is None:
            return x, list(info)[:len(b)]
        return x, list(info)[:len(b)], block_x, list(binfo)

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _lib.lib().spmv_batch_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------
# PETSc binary files and the owner_ranges split (read_petsc.cpp).
# --------------------------------------------------------------------------

def owner_ranges(size: int, n: int) -> List[int]:
    """owner_ranges (read_petsc.cpp:13-30): size + 1 boundaries splitting n
    items, the first n % size ranks one larger."""
    r = (C.c_int64 * (int(size) + 1))()
    call("spmv_owner_ranges", int(size), int(n), r)
    return list(r)


def read_petsc_binary(comm: Comm, filename: str) -> Matrix:
    """spmv::read_petsc_binary (read_petsc.cpp:32-191) for every rank of
    `comm`: the FP64 matrix of a PETSc binary file, rows and columns split by
    owner_ranges; .col_map() / .row_map() are its maps."""
    cm, rm, h = C.c_void_p(), C.c_void_p(), C.c_void_p()
    call("spmv_petsc_read_matrix", comm.handle, str(filename).encode(), C.byref(cm),
         C.byref(rm), C.byref(h))
    return _adopt_matrix(comm, cm, rm, h, np.dtype(np.float64))


def _adopt_matrix(comm: Comm, cm, rm, h, np_dtype) -> Matrix:
    """A Matrix (and its two maps) around handles the caller now owns."""
    col_map = L2GMap.__new__(L2GMap)
    col_map.comm, col_map._h = comm, cm
    row_map = L2GMap.__new__(L2GMap)
    row_map.comm, row_map._h = comm, rm
    M = Matrix.__new__(Matrix)
    M.comm, M._col_map, M._row_map, M._h = comm, col_map, row_map, h
    M.np_dtype, M.dtype = np_dtype, _DTYPES[np_dtype]
    M.nrows = [row_map.local_size(r) for r in range(comm.size)]
    M.ncols = [col_map.vec_len(r) for r in range(comm.size)]
    return M


def create_matrix(comm: Comm, blocks, nrows_local: Sequence[int], ncols_local: Sequence[int],
                  row_ghosts: Sequence[Sequence[int]],
                  col_ghosts: Sequence[Sequence[int]]) -> Matrix:
    """Matrix::create_matrix (Matrix.cpp:213-438) for every rank: blocks[r]
    = (rowptr, colind, values) with nrows_local[r] owned rows then one row
    per row_ghosts[r] entry, columns owned first then col_ghosts[r].  Ghost
    rows are summed into their owners; returns the assembled matrix, whose
    .col_map() / .row_map() are its maps."""
    P = comm.size
    rps = [np.ascontiguousarray(b[0], np.int32) for b in blocks]
    cis = [np.ascontiguousarray(b[1], np.int32) for b in blocks]
    vas = [np.ascontiguousarray(b[2]) for b in blocks]
    dts = {v.dtype for v in vas}
    if len(blocks) != P or len(dts) != 1 or next(iter(dts)) not in _DTYPES:
        raise SpmvError(_lib.ERROR_INVALID_ARGUMENT,
                        "spmv::Matrix::create_matrix - Error: one block per rank, one dtype")
    npdt = next(iter(dts))
    rg = [np.ascontiguousarray(np.asarray(g, dtype=np.int64)) for g in row_ghosts]
    cg_ = [np.ascontiguousarray(np.asarray(g, dtype=np.int64)) for g in col_ghosts]
    i64 = lambda v: (C.c_int64 * P)(*[int(t) for t in v])  # noqa: E731
    cm, rm, h = C.c_void_p(), C.c_void_p(), C.c_void_p()
    call("spmv_matrix_create_assembled", comm.handle, _DTYPES[npdt], i64(nrows_local),
         i64(ncols_local), ptr_array([a.ctypes.data for a in rps]),
         ptr_array([a.ctypes.data for a in cis]), ptr_array([a.ctypes.data for a in vas]),
         ptr_array([g.ctypes.data if len(g) else None for g in rg]), i64([len(g) for g in rg]),
         ptr_array([g.ctypes.data if len(g) else None for g in cg_]),
         i64([len(g) for g in cg_]), C.byref(cm), C.byref(rm), C.byref(h))
    return _adopt_matrix(comm, cm, rm, h, npdt)


def read_petsc_binary_vector(comm: Comm, filename: str) -> List[np.ndarray]:
    """spmv::read_petsc_binary_vector (read_petsc.cpp:193-260) for every
    rank: rank r's owner_ranges block of a PETSc binary vector file."""
    n = C.c_int64()
    call("spmv_petsc_vector_size", str(filename).encode(), C.byref(n))
    rr = owner_ranges(comm.size, n.value)
    out = [np.empty(rr[q + 1] - rr[q], dtype=np.float64) for q in range(comm.size)]
    call("spmv_petsc_read_vector", comm.handle, str(filename).encode(),
         ptr_array([v.ctypes.data if len(v) else None for v in out]))
    return out
