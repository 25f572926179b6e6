"""spmv_matrix_mult_noalloc: the product for callers that cannot allocate
device memory once they run (their memory belongs to their own pool or
allocator, and a hidden cudaMalloc could fail or stall the device).  Its
per-CTA partial sums live in a fixed device array inside the library.

Called through the C ABI and compared with spmv_matrix_mult's result on two
calls in a row (the second call runs on whatever the first left in the shared
array).  Collected last so that, should it fail, a run that stops at the first
failure has already run every other test."""
import ctypes as C

import numpy as np
import pytest
import torch

from spmv_b200 import _lib, gen
from helpers import TOL_F32, TOL_F64, abs_mult, assert_spmv_close, build, random_csr

pytestmark = pytest.mark.gpu


def noalloc(M, xs, ys):
    _lib.call("spmv_matrix_mult_noalloc", M.handle,
              _lib.ptr_array([v.data_ptr() for v in xs]),
              _lib.ptr_array([v.data_ptr() for v in ys]))


def check_against_mult(M, D, xs_host, tol):
    xs = [torch.from_numpy(x).cuda() for x in xs_host]
    ref = [y.cpu().numpy() for y in M.mult(xs)]          # existing entry point
    for _ in range(2):
        ys = [torch.full((n,), float("nan"), dtype=xs[0].dtype, device="cuda")
              for n in M.nrows]
        torch.cuda.synchronize()  # the fill runs on torch's stream
        noalloc(M, xs, ys)
        torch.cuda.synchronize()
        for q in range(D.P):
            absax = abs_mult(D.blocks[q], xs_host[q])
            assert_spmv_close(ys[q].cpu().numpy(), ref[q], absax, tol)


def test_noalloc_matches_mult_stencil(cuda_device):
    W = gen.workload("c2", scale=64)
    comm, cm, rm, M, D = build(W, 8)
    rng = np.random.default_rng(0)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)) for q in range(8)]
    check_against_mult(M, D, xs, TOL_F64)


def test_noalloc_matches_mult_skewed(cuda_device):
    rng = np.random.default_rng(1)
    A = random_csr(rng, 4000, 4000, density=0.003, long_rows=(5, 3999),
                   empty_frac=0.3)
    comm, cm, rm, M, D = build(A, 3)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(3)]
    check_against_mult(M, D, xs, TOL_F64)
    comm32, cm32, rm32, M32, D32 = build(A, 3, dtype=np.float32)
    xs32 = [x.astype(np.float32) for x in xs]
    check_against_mult(M32, D32, xs32, TOL_F32)


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
