"""Shared helpers for the parity tests."""
import json
from pathlib import Path

import numpy as np

import oracle
import spmv_b200 as S
from spmv_b200 import gen

GOLDEN = json.loads((Path(__file__).parent / "golden" / "golden.json").read_text())

# FP64 SpMV tolerance: componentwise against |A||x| (the bound that holds for
# any summation order, scaled well above n_row * eps); relative 1e-12 as the
# spec for the FP64 product states.
TOL_F64 = 1e-12
TOL_F32 = 2e-5


def assert_spmv_close(y, yref, absAx, tol):
    y, yref = np.asarray(y), np.asarray(yref)
    bound = tol * np.asarray(absAx) + 1e-300
    err = np.abs(y - yref)
    bad = np.nonzero(err > bound)[0]
    assert bad.size == 0, (bad[:5], y[bad[:5]], yref[bad[:5]], bound[bad[:5]])


def abs_mult(block, x):
    rp, ci, va = block
    return oracle.csr_mult(rp, ci, np.abs(va).astype(va.dtype), np.abs(x).astype(x.dtype))


def build(W_or_A, P, device=0, dtype=np.float64):
    """(comm, col_map, row_map, Matrix, Distributed) for a global CSR."""
    A = W_or_A.A if hasattr(W_or_A, "A") else W_or_A
    D = gen.distribute(A, P)
    comm = S.Comm(size=P, device=device)
    cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
    rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(P)])
    blocks = [(rp, ci, va.astype(dtype)) for (rp, ci, va) in D.blocks]
    M = S.Matrix(comm, blocks, cm, rm)
    D.blocks = blocks
    return comm, cm, rm, M, D


def random_csr(rng, nrows, ncols, density=0.05, long_rows=(), empty_frac=0.1):
    """CSR with sorted columns, some empty rows and optional long rows."""
    rp = [0]
    cols = []
    for i in range(nrows):
        if i in long_rows:
            k = min(ncols, max(1, int(ncols * 0.9)))
        elif rng.random() < empty_frac:
            k = 0
        else:
            k = int(rng.binomial(ncols, density))
        c = np.sort(rng.choice(ncols, size=k, replace=False)) if k else np.zeros(0, int)
        cols.extend(c.tolist())
        rp.append(len(cols))
    rp = np.array(rp, np.int32)
    cols = np.array(cols, np.int32)
    vals = rng.standard_normal(len(cols))
    return gen.CSR(rp, cols, vals, ncols)
