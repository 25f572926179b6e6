"""Complex matrices (Matrix.cpp:110-156 and the generic products of
Matrix.cpp:199-211, instantiated at Matrix.cpp:441-444): mult and transpmult
for complex64 / complex128 against the oracle's std::complex restatement.
transpmult is the plain transpose (Eigen's transpose(), no conjugation) with
the result sized cols() (the reference's MKL path sizes it rows(),
Matrix.cpp:127, 151; the generic path, followed here, sizes it cols())."""
import numpy as np
import pytest

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from helpers import random_csr

CDT = [np.complex128, np.complex64]


def complex_blocks(D, dtype, seed):
    rng = np.random.default_rng(seed)
    out = []
    for rp, ci, va in D.blocks:
        im = rng.standard_normal(len(va))
        out.append((rp, ci, (va + 1j * im).astype(dtype)))
    return out


def cvec(rng, n, dtype):
    return (rng.uniform(-1, 1, n) + 1j * rng.uniform(-1, 1, n)).astype(dtype)


@pytest.mark.parametrize("dtype", CDT)
def test_oracle_complex_product_against_numpy(dtype):
    rng = np.random.default_rng(1)
    A = random_csr(rng, 300, 200, density=0.05)
    v = cvec(rng, A.nnz, dtype)
    x = cvec(rng, 200, dtype)
    import scipy.sparse as sp
    M = sp.csr_matrix((v, A.cols, A.rowptr), shape=(300, 200))
    tol = 1e-12 if dtype == np.complex128 else 1e-5
    y = oracle.csr_mult(A.rowptr, A.cols, v, x)
    assert np.allclose(y, M @ x, rtol=tol, atol=tol)
    xt = cvec(rng, 300, dtype)
    yt = oracle.csr_transpmult(A.rowptr, A.cols, v, xt, 200)
    assert np.allclose(yt, M.T @ xt, rtol=tol, atol=tol)  # no conjugation


def build_complex(A, P, dtype, seed, device=0):
    D = gen.distribute(A, P)
    comm = S.Comm(size=P, device=device)
    cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
    rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(P)])
    blocks = complex_blocks(D, dtype, seed)
    M = S.Matrix(comm, blocks, cm, rm)
    return comm, cm, rm, M, blocks


def test_complex_matrix_host_only_create_and_mat():
    # Creation and Matrix::mat() need no GPU.
    W = gen.workload("c1", 64)
    comm, cm, rm, M, blocks = build_complex(W.A, 2, np.complex128, 3, device=-1)
    for r in range(2):
        rp, ci, va = M.mat(r)
        assert np.array_equal(va, blocks[r][2])


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", CDT)
@pytest.mark.parametrize("cfg,P", [("c2", 3), ("c1", 1)])
@pytest.mark.parametrize("kernel", ["auto", "sell", "vector"])
def test_complex_mult_and_transpmult(cuda_device, dtype, cfg, P, kernel):
    W = gen.workload(cfg, 16 if cfg == "c2" else 48)
    comm, cm, rm, M, blocks = build_complex(W.A, P, dtype, 5)
    M.set_kernel(kernel)
    rng = np.random.default_rng(9)
    xs = [cvec(rng, cm.vec_len(q), dtype) for q in range(P)]
    ys = M.mult(xs)
    real = np.float64 if dtype == np.complex128 else np.float32
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    for q in range(P):
        rp, ci, va = blocks[q]
        yref = oracle.csr_mult(rp, ci, va, xs[q])
        if kernel in ("auto", "sell"):  # SELL-32: storage order, bitwise
            assert np.array_equal(ys[q], yref)
        else:
            bound = tol * np.abs(oracle.csr_mult(rp, ci, np.abs(va).astype(dtype),
                                                 np.abs(xs[q]).astype(dtype))) + 1e-300
            assert np.all(np.abs(ys[q] - yref) <= bound)
    # transpmult: y[r] has ncols[r] entries; SELL over A^T sums each column
    # of A in ascending row order, the reference's scatter order.
    zs = [cvec(rng, rm.local_size(q), dtype) for q in range(P)]
    ts = M.transpmult(zs)
    for q in range(P):
        rp, ci, va = blocks[q]
        tref = oracle.csr_transpmult(rp, ci, va, zs[q], cm.vec_len(q))
        assert ts[q].shape == (cm.vec_len(q),)
        assert np.array_equal(ts[q], tref)
    assert real  # dtype bookkeeping


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", CDT)
def test_complex_uneven_rows(cuda_device, dtype):
    # Skewed rows: merge-path is real only, so the complex product runs
    # vector CSR (within tolerance of the oracle).
    rng = np.random.default_rng(2)
    A = random_csr(rng, 2000, 2000, density=0.003, long_rows=(5, 1999))
    comm, cm, rm, M, blocks = build_complex(A, 2, dtype, 8)
    xs = [cvec(rng, cm.vec_len(q), dtype) for q in range(2)]
    ys = M.mult(xs)
    tol = 1e-12 if dtype == np.complex128 else 2e-5
    for q in range(2):
        rp, ci, va = blocks[q]
        yref = oracle.csr_mult(rp, ci, va, xs[q])
        bound = tol * np.abs(oracle.csr_mult(rp, ci, np.abs(va).astype(dtype),
                                             np.abs(xs[q]).astype(dtype))) + 1e-300
        assert np.all(np.abs(ys[q] - yref) <= bound)
    ts = M.transpmult([cvec(rng, rm.local_size(q), dtype) for q in range(2)])
    assert all(np.all(np.isfinite(t)) for t in ts)


@pytest.mark.gpu
def test_complex_matrix_rejected_by_real_only_calls(cuda_device):
    W = gen.workload("c1", 64)
    comm, cm, rm, M, blocks = build_complex(W.A, 1, np.complex128, 4)
    b = [np.ones(rm.local_size(0))]
    with pytest.raises(S.SpmvError, match="float64"):
        S.cg(comm, M, b, 10, 1e-8)
