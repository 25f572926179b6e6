"""Seeded synthetic workloads and their row-block distribution.

`distribute` splits a global CSR into the local blocks the reference's demos
build (CreateA.cpp:77-108): rank r owns the rows owner_ranges gives it
(CreateA.cpp:12-29), its ghosts are the sorted distinct columns outside its
range, owned columns are renumbered from 0 and ghost column g becomes
local_size + (position of g among the ghosts), and each row is sorted by
local column, as Eigen's setFromTriplets leaves it.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Optional

import numpy as np

PKG = Path(__file__).resolve().parent
GEN_PATH = PKG / "libspmv_gen.so"

_gen = None


def gen_lib():
    global _gen
    if _gen is None:
        if not GEN_PATH.exists():
            raise ImportError(f"{GEN_PATH} is missing: run `python -m spmv_b200.build`")
        L = C.CDLL(str(GEN_PATH))
        h = C.POINTER(C.c_void_p)
        L.spmv_gen_last_error.restype = C.c_char_p
        L.spmv_gen_uniform.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double,
                                       C.c_void_p, C.c_int64]
        L.spmv_gen_normal.argtypes = L.spmv_gen_uniform.argtypes
        L.spmv_gen_laplace2d.argtypes = [C.c_int64, C.c_int64, h]
        L.spmv_gen_laplace3d.argtypes = [C.c_int64, h]
        L.spmv_gen_laplace3d_27pt.argtypes = [C.c_int64, C.c_uint64, C.c_double, h]
        L.spmv_gen_grid2d_softplus.argtypes = [C.c_int64, C.c_int64, C.c_uint64,
                                               C.c_double, C.c_double, h]
        L.spmv_gen_knn_laplacian.argtypes = [C.c_int64, C.c_int, C.c_uint64, C.c_uint64,
                                             C.c_double, h]
        L.spmv_gen_create_a.argtypes = [C.c_int64, h]
        L.spmv_gen_csr_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 3
        L.spmv_gen_csr_arrays.argtypes = [C.c_void_p, C.POINTER(C.POINTER(C.c_int32)),
                                          C.POINTER(C.POINTER(C.c_int32)),
                                          C.POINTER(C.POINTER(C.c_double))]
        L.spmv_gen_csr_aux.argtypes = [C.c_void_p, C.POINTER(C.c_double),
                                       C.POINTER(C.POINTER(C.c_int64)),
                                       C.POINTER(C.c_int64),
                                       C.POINTER(C.POINTER(C.c_double)),
                                       C.POINTER(C.c_int64)]
        L.spmv_gen_csr_free.argtypes = [C.c_void_p]
        _gen = L
    return _gen


@dataclass
class CSR:
    """Global CSR (int32 indices, sorted columns per row)."""
    rowptr: np.ndarray
    cols: np.ndarray
    vals: np.ndarray
    ncols: int
    scalar: float = 0.0
    aux_i64: Optional[np.ndarray] = None
    aux_f64: Optional[np.ndarray] = None

    @property
    def nrows(self) -> int:
        return len(self.rowptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.rowptr[-1])

    def scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.vals, self.cols, self.rowptr),
                             shape=(self.nrows, self.ncols))


def _take(fn, *args) -> CSR:
    L = gen_lib()
    h = C.c_void_p()
    if fn(*args, C.byref(h)) != 0:
        raise RuntimeError(L.spmv_gen_last_error().decode())
    try:
        n, m, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        L.spmv_gen_csr_info(h, C.byref(n), C.byref(m), C.byref(nnz))
        rp, ci, va = (C.POINTER(C.c_int32)(), C.POINTER(C.c_int32)(),
                      C.POINTER(C.c_double)())
        L.spmv_gen_csr_arrays(h, C.byref(rp), C.byref(ci), C.byref(va))
        s = C.c_double()
        pi, ni, pf, nf = (C.POINTER(C.c_int64)(), C.c_int64(), C.POINTER(C.c_double)(),
                          C.c_int64())
        L.spmv_gen_csr_aux(h, C.byref(s), C.byref(pi), C.byref(ni), C.byref(pf),
                           C.byref(nf))
        arr = np.ctypeslib.as_array
        out = CSR(arr(rp, (n.value + 1,)).copy(),
                  arr(ci, (nnz.value,)).copy() if nnz.value else np.zeros(0, np.int32),
                  arr(va, (nnz.value,)).copy() if nnz.value else np.zeros(0),
                  m.value, s.value,
                  arr(pi, (ni.value,)).copy() if ni.value else None,
                  arr(pf, (nf.value,)).copy() if nf.value else None)
    finally:
        L.spmv_gen_csr_free(h)
    return out


def laplace2d(nx: int, ny: int) -> CSR:
    return _take(gen_lib().spmv_gen_laplace2d, nx, ny)


def laplace3d(n: int) -> CSR:
    return _take(gen_lib().spmv_gen_laplace3d, n)


def laplace3d_27pt(n: int, seed: int, shift: float = 1e-3) -> CSR:
    return _take(gen_lib().spmv_gen_laplace3d_27pt, n, seed, shift)


def grid2d_softplus(nx: int, ny: int, seed: int, sigma: float = 0.5,
                    shift: float = 1e-3) -> CSR:
    return _take(gen_lib().spmv_gen_grid2d_softplus, nx, ny, seed, sigma, shift)


def knn_laplacian(n: int, k: int, seed: int, sys: int, shift: float = 1e-2) -> CSR:
    return _take(gen_lib().spmv_gen_knn_laplacian, n, k, seed, sys, shift)


def create_a(N: int) -> CSR:
    return _take(gen_lib().spmv_gen_create_a, N)


def uniform(seed: int, stream: int, n: int, lo: float = -1.0, hi: float = 1.0):
    out = np.empty(n, np.float64)
    gen_lib().spmv_gen_uniform(seed, stream, lo, hi, out.ctypes.data, n)
    return out


def normal(seed: int, stream: int, n: int, mean: float = 0.0, std: float = 1.0):
    out = np.empty(n, np.float64)
    gen_lib().spmv_gen_normal(seed, stream, mean, std, out.ctypes.data, n)
    return out


def owner_ranges(size: int, N: int) -> np.ndarray:
    """Row ranges of `size` ranks over N rows: the first N % size ranks get
    one extra row (the split of CreateA.cpp:12-29)."""
    n, r = divmod(N, size)
    return np.array([k * (n + 1) if k < r else k * n + r for k in range(size + 1)],
                    dtype=np.int64)


@dataclass
class Distributed:
    """Row-block distribution of a square global matrix over P ranks."""
    ranges: np.ndarray
    local_sizes: List[int]
    ghosts: List[np.ndarray]
    blocks: List[tuple] = field(default_factory=list)  # (rowptr, cols, vals)

    @property
    def P(self) -> int:
        return len(self.local_sizes)


def distribute(A: CSR, P: int) -> Distributed:
    ranges = owner_ranges(P, A.nrows)
    sizes, ghosts, blocks = [], [], []
    for q in range(P):
        r0, r1 = int(ranges[q]), int(ranges[q + 1])
        M = r1 - r0
        a, b = int(A.rowptr[r0]), int(A.rowptr[r1])
        rp = (A.rowptr[r0:r1 + 1] - a).astype(np.int32)
        cols = A.cols[a:b].astype(np.int64)
        vals = A.vals[a:b]
        is_g = (cols < r0) | (cols >= r1)
        g = np.unique(cols[is_g])
        local = np.where(is_g, M + np.searchsorted(g, cols), cols - r0)
        if is_g.any():
            # Re-sort rows that hold ghosts by local column (owned first).
            row_id = np.repeat(np.arange(M, dtype=np.int64), np.diff(rp))
            order = np.lexsort((local, row_id))
            local = local[order]
            vals = vals[order]
        sizes.append(M)
        ghosts.append(g.astype(np.int64))
        blocks.append((rp, local.astype(np.int32), np.ascontiguousarray(vals)))
    return Distributed(ranges, sizes, ghosts, blocks)


# ---------------------------------------------------------------------------
# The five workloads (all seeded, synthetic)
# ---------------------------------------------------------------------------
@dataclass
class Workload:
    name: str
    A: CSR
    P: int
    b: np.ndarray
    rtol: float
    extra: dict = field(default_factory=dict)


def workload(name: str, scale: int = 0) -> Workload:
    """c1..c5 at full size (scale=0) or a reduced size for fast tests.

    c1  2D 5-point Laplacian 512^2, 1 rank, b ~ U[-1,1] seed 0, rtol 1e-8
    c2  3D 7-point Laplacian 128^3, 8 ranks, b ~ U[-1,1] seed 1, rtol 1e-8
    c3  27-point lognormal-weighted Laplacian 160^3 (+1e-3 I), b ~ N(0,1)
        seed 2, rtol 1e-10
    c5  1024^2 grid graph, w = softplus(theta), theta ~ N(0, 0.5) (0.5 is the
        standard deviation), +1e-3 I, b, x* ~ N(0,1) seed 4
    """
    if name == "c1":
        n = 512 if scale == 0 else scale
        A = laplace2d(n, n)
        return Workload(name, A, 1, uniform(0, 100, A.nrows), 1e-8)
    if name == "c2":
        n = 128 if scale == 0 else scale
        A = laplace3d(n)
        return Workload(name, A, 8, uniform(1, 100, A.nrows), 1e-8)
    if name == "c3":
        n = 160 if scale == 0 else scale
        A = laplace3d_27pt(n, 2, 1e-3)
        return Workload(name, A, 1, normal(2, 100, A.nrows), 1e-10)
    if name == "c5":
        n = 1024 if scale == 0 else scale
        A = grid2d_softplus(n, n, 4, 0.5, 1e-3)
        return Workload(name, A, 1, normal(4, 100, A.nrows), 1e-10,
                        {"xstar": normal(4, 101, A.nrows)})
    raise ValueError(name)


def c4_sizes(count: int = 256, lo: int = 4096, hi: int = 131072, seed: int = 3):
    """System sizes of the batched workload: integers uniform in [lo, hi]."""
    u = uniform(seed, 200, count, 0.0, 1.0)
    return [int(lo + int(v * (hi - lo + 1))) for v in u]


def c4_systems(count: int = 256, lo: int = 4096, hi: int = 131072, seed: int = 3,
               k: int = 12, shift: float = 1e-2):
    """The batched workload: `count` k-NN graph Laplacians over uniform points
    in the unit cube (w = exp(-d^2/h^2), h = mean k-NN distance per system,
    +shift on the diagonal), with b ~ N(0,1) per system (stream 300 + i).
    Returns a list of (CSR, b)."""
    out = []
    for i, n in enumerate(c4_sizes(count, lo, hi, seed)):
        A = knn_laplacian(n, k, seed, i, shift)
        out.append((A, normal(seed, 300 + i, n)))
    return out


def c4_block_rhs(n: int, nrhs: int = 32, seed: int = 3):
    """The batched workload's block of right-hand sides for system 0:
    n x nrhs, row-major, column l ~ N(0,1) from stream 400 + l."""
    return np.ascontiguousarray(np.stack([normal(seed, 400 + l, n) for l in range(nrhs)],
                                         axis=1))


def grid_assembly_5pt(nx: int, P: int):
    """Input of create_matrix (Matrix.cpp:213-438) for a 5-point assembly on
    an nx x nx node grid over P ranks: rank r lists the rows of its own nodes
    and of the next grid line (ghost rows owned by rank r + 1), each coupling
    entered twice (from two elements; the assembly sums repeats), value 0.5.
    Returns (blocks, nrows_local, row_ghosts, col_ghosts) as create_matrix
    takes them."""
    nodes = nx * nx
    rr = owner_ranges(P, nodes)
    bl, nrl, rgs, cgs = [], [], [], []
    for r in range(P):
        r0, r1 = rr[r], rr[r + 1]
        j0, j1 = r0 // nx, min((r1 + nx - 1) // nx, nx - 1)
        rows = np.arange(j0 * nx, min((j1 + 1) * nx, nodes))
        ghost_rows = rows[(rows < r0) | (rows >= r1)]
        rowlist = np.concatenate([np.arange(r0, r1), ghost_rows])
        cols, rptr = [], [0]
        for gr in rowlist:
            i, j = gr % nx, gr // nx
            nb = [gr] + [q for q, ok in ((gr - 1, i > 0), (gr + 1, i < nx - 1),
                                         (gr - nx, j > 0), (gr + nx, j < nx - 1)) if ok]
            cols.extend(nb + nb)
            rptr.append(len(cols))
        cols = np.array(cols, np.int64)
        gh = np.unique(cols[(cols < r0) | (cols >= r1)])
        loc = np.where((cols >= r0) & (cols < r1), cols - r0,
                       (r1 - r0) + np.searchsorted(gh, cols))
        bl.append((np.array(rptr, np.int32), loc.astype(np.int32), np.full(len(cols), 0.5)))
        nrl.append(int(r1 - r0))
        rgs.append(ghost_rows.astype(np.int64))
        cgs.append(gh)
    return bl, nrl, rgs, cgs
