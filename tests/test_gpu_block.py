"""Several right-hand sides: the block product equals k single products, and
block CG solves k systems at once with per-column stopping, matching k
separate spmv::cg solves."""
import numpy as np
import pytest
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from spmv_b200.core import cg_block
from helpers import TOL_F64, abs_mult, assert_spmv_close, build, random_csr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("k", [1, 3, 8, 32])
def test_mult_block_equals_single_products(cuda_device, k):
    rng = np.random.default_rng(k)
    A = random_csr(rng, 3000, 3000, density=0.004, long_rows=(9,))
    comm, cm, rm, M, D = build(A, 3)
    X = [rng.standard_normal((cm.vec_len(q), k)) for q in range(3)]
    for dev in (False, True):
        Xi = [torch.from_numpy(x).cuda() for x in X] if dev else X
        Y = M.mult_block(Xi)
        Y = [y.cpu().numpy() for y in Y] if dev else Y
        for q in range(3):
            rp, ci, va = D.blocks[q]
            for l in range(k):
                x = np.ascontiguousarray(X[q][:, l])
                assert_spmv_close(Y[q][:, l], oracle.csr_mult(rp, ci, va, x),
                                  abs_mult(D.blocks[q], x), TOL_F64)


@pytest.mark.parametrize("k", [2, 32])
def test_block_cg_matches_single_solves(cuda_device, k):
    W = gen.workload("c2", 24)
    comm, cm, rm, M, D = build(W, 8)
    rng = np.random.default_rng(5)
    Bg = rng.uniform(-1, 1, (W.A.nrows, k))
    Bg[:, -1] *= 1e-3        # a differently scaled column converges separately
    B = [np.ascontiguousarray(Bg[D.ranges[q]:D.ranges[q + 1]]) for q in range(8)]
    X, info = cg_block(comm, M, B, 10000, 1e-8)
    for q in range(8):
        assert np.all(X[q][D.local_sizes[q]:] == 0.0)
    Xg = np.concatenate([X[q][:D.local_sizes[q]] for q in range(8)])
    Sp = W.A.scipy()
    for l in range(k):
        assert info[l].status == 0
        b = np.ascontiguousarray(Bg[:, l])
        rel = np.linalg.norm(b - Sp @ Xg[:, l]) / np.linalg.norm(b)
        assert rel < 1.5e-8, (l, rel)
        xs, ks = S.cg(comm, M, [np.ascontiguousarray(B[q][:, l]) for q in range(8)],
                      10000, 1e-8)
        assert abs(info[l].iterations - ks) <= 2
        xsg = np.concatenate([xs[q][:D.local_sizes[q]] for q in range(8)])
        assert np.linalg.norm(Xg[:, l] - xsg) <= 1e-9 * np.linalg.norm(xsg)


def test_block_cg_c4_system_32_rhs(cuda_device):
    # The batched workload's system with 32 right-hand sides (k-NN Laplacian).
    A = gen.knn_laplacian(20000, 12, 3, 0, 1e-2)
    comm = S.Comm(size=1, device=0)
    cm = S.L2GMap(comm, [A.nrows], [[]])
    M = S.Matrix(comm, [(A.rowptr, A.cols, A.vals)], cm, cm)
    Bt = torch.from_numpy(np.stack([gen.normal(3, 400 + l, A.nrows) for l in range(32)],
                                   axis=1)).cuda()
    X, info = cg_block(comm, M, [Bt.contiguous()], 20000, 1e-10)
    Xh, Bh = X[0].cpu().numpy(), Bt.cpu().numpy()
    Sp = A.scipy()
    rel = np.linalg.norm(Bh - Sp @ Xh, axis=0) / np.linalg.norm(Bh, axis=0)
    assert np.all(rel < 1.5e-10), rel.max()
    assert all(i.status == 0 for i in info)
