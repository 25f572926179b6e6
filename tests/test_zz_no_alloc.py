"""spmv_matrix_mult_noalloc: the product for callers that cannot allocate
device memory once they run (their memory belongs to their own pool or
allocator, and a hidden cudaMalloc could fail or stall the device).  Its
per-CTA partial sums live in a fixed device array inside the library.

Called through the C ABI, checked against the oracle's restatement of
Matrix::operator* (Matrix.cpp:199-204) within the product tolerance, and
bitwise against spmv_matrix_mult when that entry point also runs the
merge-path kernel, on two calls in a row (the second call runs on whatever
the first left in the shared array), and after a call on a larger matrix
that used more of the array.  Collected last so that, should it fail, a run
that stops at the first failure has already run every other test."""
import numpy as np
import pytest
import torch

import oracle
from spmv_b200 import _lib, gen
from helpers import TOL_F32, TOL_F64, abs_mult, assert_spmv_close, build, random_csr

pytestmark = pytest.mark.gpu


def noalloc(M, xs, ys):
    _lib.call("spmv_matrix_mult_noalloc", M.handle,
              _lib.ptr_array([v.data_ptr() for v in xs]),
              _lib.ptr_array([v.data_ptr() for v in ys]))


def run_noalloc(M, xs):
    ys = [torch.full((n,), float("nan"), dtype=xs[0].dtype, device="cuda")
          for n in M.nrows]
    torch.cuda.synchronize()  # the fill runs on torch's stream
    noalloc(M, xs, ys)
    torch.cuda.synchronize()
    return [y.cpu().numpy() for y in ys]


def check(M, D, xs_host, tol):
    """Two calls in a row: each within tol of the oracle and bitwise equal to
    spmv_matrix_mult on the merge-path kernel."""
    xs = [torch.from_numpy(x).cuda() for x in xs_host]
    M.set_kernel("merge")
    ref = [y.cpu().numpy() for y in M.mult(xs)]          # existing entry point
    M.set_kernel("auto")
    for _ in range(2):
        ys = run_noalloc(M, xs)
        for q in range(D.P):
            rp, ci, va = D.blocks[q]
            yo = oracle.csr_mult(rp, ci, va, xs_host[q])
            assert_spmv_close(ys[q], yo, abs_mult(D.blocks[q], xs_host[q]), tol)
            np.testing.assert_array_equal(ys[q], ref[q])


def test_noalloc_matches_oracle_stencil(cuda_device):
    W = gen.workload("c2", scale=64)
    comm, cm, rm, M, D = build(W, 8)
    rng = np.random.default_rng(0)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)) for q in range(8)]
    check(M, D, xs, TOL_F64)


def test_noalloc_matches_oracle_skewed(cuda_device):
    rng = np.random.default_rng(1)
    A = random_csr(rng, 4000, 4000, density=0.003, long_rows=(5, 3999),
                   empty_frac=0.3)
    comm, cm, rm, M, D = build(A, 3)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(3)]
    check(M, D, xs, TOL_F64)
    comm32, cm32, rm32, M32, D32 = build(A, 3, dtype=np.float32)
    xs32 = [x.astype(np.float32) for x in xs]
    check(M32, D32, xs32, TOL_F32)


def test_noalloc_small_after_large(cuda_device):
    # A product over ~8,200 tiles leaves its partial sums in the shared array;
    # a smaller matrix run next must not pick any of them up.
    rng = np.random.default_rng(2)
    big = gen.workload("c2", scale=128)           # 128^3 rows: ~8,100 tiles
    comm_b, cm_b, rm_b, Mb, Db = build(big, 8)
    xb = [torch.from_numpy(rng.uniform(-1, 1, cm_b.vec_len(q))).cuda() for q in range(8)]
    run_noalloc(Mb, xb)
    A = random_csr(rng, 3000, 3000, density=0.004, long_rows=(7,), empty_frac=0.2)
    comm, cm, rm, M, D = build(A, 2)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(2)]
    check(M, D, xs, TOL_F64)


def test_noalloc_rejects_matrices_over_its_limit(cuda_device):
    # 16384 tiles of 2048 rows + nonzeros is the maximum; one more row is over.
    n = 16384 * 2048 + 1
    rp = np.zeros(n + 1, np.int32)
    A = gen.CSR(rp, np.zeros(0, np.int32), np.zeros(0), n)
    comm, cm, rm, M, D = build(A, 1)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    y = torch.zeros(n, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.SpmvError) as e:
        noalloc(M, [x], [y])
    assert e.value.status == _lib.ERROR_INVALID_ARGUMENT
    assert "exceed the maximum" in str(e.value)
