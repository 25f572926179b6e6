"""Matrix::operator* and transpmult on the GPU against the oracle's
restatement of the reference's Eigen products (Matrix.cpp:199-211)."""
import numpy as np
import pytest
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from helpers import (TOL_F32, TOL_F64, abs_mult, assert_spmv_close, build,
                     random_csr)

pytestmark = pytest.mark.gpu


def check_mult(M, D, xs, tol, device=False):
    if device:
        xt = [torch.from_numpy(x).cuda() for x in xs]
        ys = [y.cpu().numpy() for y in M.mult(xt)]
    else:
        ys = M.mult(xs)
    for q in range(D.P):
        rp, ci, va = D.blocks[q]
        yref = oracle.csr_mult(rp, ci, va, xs[q])
        assert_spmv_close(ys[q], yref, abs_mult(D.blocks[q], xs[q]), tol)
    return ys


@pytest.mark.parametrize("cfg,P", [("c1", 1), ("c2", 8), ("c2", 3), ("c1", 2)])
def test_mult_matches_oracle(cuda_device, cfg, P):
    W = gen.workload(cfg)
    comm, cm, rm, M, D = build(W, P)
    rng = np.random.default_rng(0)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)) for q in range(P)]
    y_host = check_mult(M, D, xs, TOL_F64)
    y_dev = check_mult(M, D, xs, TOL_F64, device=True)
    for a, b in zip(y_host, y_dev):
        assert np.array_equal(a, b)  # same kernel, same order: bitwise


def test_mult_float32(cuda_device):
    W = gen.workload("c2", scale=48)
    comm, cm, rm, M, D = build(W, 4, dtype=np.float32)
    rng = np.random.default_rng(1)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)).astype(np.float32) for q in range(4)]
    check_mult(M, D, xs, TOL_F32)
    check_mult(M, D, xs, TOL_F32, device=True)


@pytest.mark.parametrize("width", [1, 2, 4, 8, 16, 32])
@pytest.mark.parametrize("block", [128, 256, 512])
def test_every_width_and_block(cuda_device, width, block):
    rng = np.random.default_rng(width * 1000 + block)
    A = random_csr(rng, 3001, 3001, density=0.004, long_rows=(7, 2500))
    comm, cm, rm, M, D = build(A, 3)
    M.set_kernel("vector", width, block)
    assert M.get_kernel() == ("vector", width, block)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(3)]
    check_mult(M, D, xs, TOL_F64)


@pytest.mark.parametrize("seed", range(6))
def test_ragged_random_matrices(cuda_device, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(1, 4000))
    P = int(rng.integers(1, 9))
    A = random_csr(rng, n, n, density=float(rng.uniform(0.0, 0.02)),
                   long_rows=tuple(rng.integers(0, n, size=2)),
                   empty_frac=float(rng.uniform(0, 0.5)))
    comm, cm, rm, M, D = build(A, min(P, n))
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(D.P)]
    check_mult(M, D, xs, TOL_F64)
    M32 = S.Matrix(comm, [(rp, ci, va.astype(np.float32)) for rp, ci, va in D.blocks],
                   cm, rm)
    ys = M32.mult([x.astype(np.float32) for x in xs])
    for q in range(D.P):
        rp, ci, va = D.blocks[q]
        yref = oracle.csr_mult(rp, ci, va.astype(np.float32), xs[q].astype(np.float32))
        assert_spmv_close(ys[q], yref, abs_mult(D.blocks[q], xs[q]).astype(np.float32),
                          TOL_F32)


def test_empty_and_zero_row_ranks(cuda_device):
    # A rank with no rows, a matrix with no entries, a 1x1 matrix.
    comm = S.Comm(size=3, device=0)
    cm = S.L2GMap(comm, [0, 2, 1], [[], [], []])
    blocks = [(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0)),
              (np.array([0, 0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0)),
              (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([2.5]))]
    M = S.Matrix(comm, blocks, cm, cm)
    ys = M.mult([np.zeros(0), np.ones(2), np.array([3.0])])
    assert ys[0].size == 0 and np.array_equal(ys[1], [0, 0]) and ys[2][0] == 7.5


@pytest.mark.parametrize("cfg,P", [("c2", 8), ("c1", 1)])
def test_transpmult_matches_oracle(cuda_device, cfg, P):
    W = gen.workload(cfg, scale=40 if cfg == "c2" else 0)
    comm, cm, rm, M, D = build(W, P)
    rng = np.random.default_rng(2)
    xs = [rng.uniform(-1, 1, D.local_sizes[q]) for q in range(P)]
    ys = M.transpmult(xs)
    for q in range(P):
        rp, ci, va = D.blocks[q]
        n = cm.vec_len(q)
        yref = oracle.csr_transpmult(rp, ci, va, xs[q], n)
        absx = oracle.csr_transpmult(rp, ci, np.abs(va), np.abs(xs[q]), n)
        assert ys[q].shape == (n,)
        assert_spmv_close(ys[q], yref, absx, TOL_F64)


def test_transpmult_ragged(cuda_device):
    rng = np.random.default_rng(9)
    A = random_csr(rng, 1500, 1500, density=0.01, long_rows=(3,))
    comm, cm, rm, M, D = build(A, 4)
    xs = [rng.standard_normal(D.local_sizes[q]) for q in range(4)]
    ys = M.transpmult(xs)
    for q in range(4):
        rp, ci, va = D.blocks[q]
        n = cm.vec_len(q)
        assert_spmv_close(ys[q], oracle.csr_transpmult(rp, ci, va, xs[q], n),
                          oracle.csr_transpmult(rp, ci, np.abs(va), np.abs(xs[q]), n),
                          TOL_F64)


def test_set_values_keeps_pattern(cuda_device):
    W = gen.workload("c1", scale=64)
    comm, cm, rm, M, D = build(W, 2)
    new = [va * 2.0 for (_, _, va) in D.blocks]
    M.set_values(new)
    D.blocks = [(rp, ci, v) for (rp, ci, _), v in zip(D.blocks, new)]
    rng = np.random.default_rng(3)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)) for q in range(2)]
    check_mult(M, D, xs, TOL_F64)


@pytest.mark.parametrize("seed", range(5))
def test_merge_path_matches_oracle(cuda_device, seed):
    rng = np.random.default_rng(500 + seed)
    n = int(rng.integers(50, 5000))
    A = random_csr(rng, n, n, density=float(rng.uniform(0.0, 0.01)),
                   long_rows=tuple(rng.integers(0, n, size=3)),
                   empty_frac=float(rng.uniform(0, 0.6)))
    P = int(rng.integers(1, 5))
    comm, cm, rm, M, D = build(A, P)
    M.set_kernel("merge")
    assert M.get_kernel()[0] == "merge"
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(P)]
    ys1 = check_mult(M, D, xs, TOL_F64)
    ys2 = M.mult(xs)
    assert all(np.array_equal(a, b) for a, b in zip(ys1, ys2))  # reproducible
    xt = [rng.standard_normal(D.local_sizes[q]) for q in range(P)]
    yt = M.transpmult(xt)
    for q in range(P):
        rp, ci, va = D.blocks[q]
        nc = cm.vec_len(q)
        assert_spmv_close(yt[q], oracle.csr_transpmult(rp, ci, va, xt[q], nc),
                          oracle.csr_transpmult(rp, ci, np.abs(va), np.abs(xt[q]), nc),
                          TOL_F64)


def test_auto_picks_merge_for_a_dense_row(cuda_device):
    n = 20000
    rng = np.random.default_rng(7)
    lens = np.full(n, 3)
    lens[17] = n  # one full row
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cols = np.concatenate([np.sort(rng.choice(n, size=k, replace=False)) for k in lens])
    A = gen.CSR(rp, cols.astype(np.int32), rng.standard_normal(rp[-1]), n)
    comm, cm, rm, M, D = build(A, 1)
    assert M.get_kernel()[0] == "merge"
    xs = [rng.standard_normal(n)]
    check_mult(M, D, xs, TOL_F64)
    M32 = S.Matrix(comm, [(rp, cols.astype(np.int32), D.blocks[0][2].astype(np.float32))],
                   cm, rm)
    y32 = M32.mult([xs[0].astype(np.float32)])[0]
    yref = oracle.csr_mult(rp, cols.astype(np.int32), D.blocks[0][2].astype(np.float32),
                           xs[0].astype(np.float32))
    assert_spmv_close(y32, yref, abs_mult(D.blocks[0], xs[0]).astype(np.float32), TOL_F32)


@pytest.mark.parametrize("cfg,P", [("c1", 1), ("c2", 8), ("c3", 1)])
def test_sell_is_bitwise_equal_to_oracle(cuda_device, cfg, P):
    # SELL-32 sums each row in storage order, like the reference's row loop.
    W = gen.workload(cfg, scale=0 if cfg != "c3" else 40)
    comm, cm, rm, M, D = build(W, P)
    assert M.get_kernel()[0] == "sell"  # chosen automatically for stencils
    rng = np.random.default_rng(4)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)) for q in range(P)]
    ys = M.mult(xs)
    for q in range(P):
        rp, ci, va = D.blocks[q]
        assert np.array_equal(ys[q], oracle.csr_mult(rp, ci, va, xs[q]))
    M32 = S.Matrix(comm, [(rp, ci, va.astype(np.float32)) for rp, ci, va in D.blocks],
                   cm, rm)
    ys32 = M32.mult([x.astype(np.float32) for x in xs])
    for q in range(P):
        rp, ci, va = D.blocks[q]
        assert np.array_equal(ys32[q], oracle.csr_mult(rp, ci, va.astype(np.float32),
                                                       xs[q].astype(np.float32)))


@pytest.mark.parametrize("cfg,P,width", [("c1", 1, 8), ("c2", 8, 4), ("c2", 3, 8), ("c3", 1, 8),
                                         ("c1", 2, 5), ("c2", 8, 7), ("c3", 1, 9), ("c3", 3, 9)])
def test_staged_is_bitwise_equal_to_oracle(cuda_device, cfg, P, width):
    # The staged SELL-32 product (tiles streamed into shared memory by bulk
    # copies) also sums rows in storage order; widths 5, 7 and 9 take the
    # unmasked path on the 5-, 7- and 27-point stencils' full slices.
    W = gen.workload(cfg, scale=0 if cfg != "c3" else 40)
    comm, cm, rm, M, D = build(W, P)
    M.set_kernel("staged", width)
    assert M.get_kernel()[:2] == ("staged", width)
    rng = np.random.default_rng(5)
    xs = [rng.uniform(-1, 1, cm.vec_len(q)) for q in range(P)]
    for _ in range(2):  # a second call reuses the tile table
        ys = M.mult(xs)
        for q in range(P):
            rp, ci, va = D.blocks[q]
            assert np.array_equal(ys[q], oracle.csr_mult(rp, ci, va, xs[q]))
    comm.synchronize()  # no bounded wait timed out
    M32 = S.Matrix(comm, [(rp, ci, va.astype(np.float32)) for rp, ci, va in D.blocks],
                   cm, rm)
    M32.set_kernel("staged", width)
    ys32 = M32.mult([x.astype(np.float32) for x in xs])
    for q in range(P):
        rp, ci, va = D.blocks[q]
        assert np.array_equal(ys32[q], oracle.csr_mult(rp, ci, va.astype(np.float32),
                                                       xs[q].astype(np.float32)))


def test_staged_wide_rows_fall_back(cuda_device):
    # A slice wider than one stage cannot be staged: the product runs SELL-32
    # from registers and still matches the oracle.
    rng = np.random.default_rng(11)
    A = random_csr(rng, 3000, 3000, density=0.002, long_rows=(3, 2900))
    comm, cm, rm, M, D = build(A, 2)
    M.set_kernel("staged", 8)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(2)]
    ys = M.mult(xs)
    for q in range(2):
        rp, ci, va = D.blocks[q]
        assert np.array_equal(ys[q], oracle.csr_mult(rp, ci, va, xs[q]))


@pytest.mark.parametrize("width", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("block", [128, 256, 512])
def test_sell_every_width_and_block(cuda_device, width, block):
    rng = np.random.default_rng(width * 7 + block)
    A = random_csr(rng, 2999, 2999, density=0.004, long_rows=(7, 2500))
    comm, cm, rm, M, D = build(A, 3)
    M.set_kernel("sell", width, block)
    assert M.get_kernel() == ("sell", width, block)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(3)]
    ys = M.mult(xs)
    for q in range(3):
        rp, ci, va = D.blocks[q]
        assert np.array_equal(ys[q], oracle.csr_mult(rp, ci, va, xs[q]))


def test_set_values_reaches_every_kernel_copy(cuda_device):
    # New values must reach the SELL copy and the solvers' graphs, not only
    # the CSR (one matrix re-used with changing values, as in a parameter
    # sweep or finite differences).
    W = gen.workload("c1", scale=48)
    comm, cm, rm, M, D = build(W, 1)
    assert M.get_kernel()[0] == "sell"
    b = [W.b.copy()]
    x1, k1 = S.cg(comm, M, b, 10000, 1e-10)
    xm1, _ = S.cg_mixed(comm, M, b, 10000, 1e-10)
    M.set_values([D.blocks[0][2] * 4.0])
    xs = [np.random.default_rng(0).standard_normal(cm.vec_len(0))]
    y = M.mult(xs)[0]
    rp, ci, va = D.blocks[0]
    assert np.array_equal(y, oracle.csr_mult(rp, ci, va * 4.0, xs[0]))
    x2, k2 = S.cg(comm, M, b, 10000, 1e-10)
    xm2, _ = S.cg_mixed(comm, M, b, 10000, 1e-10)
    # Each solver workspace re-picks its product by timing after new values,
    # so the two solves may sum rows in different orders: both solutions are
    # within 1e-10 relative residual, close but not bitwise equal.
    assert np.linalg.norm(x2[0] * 4.0 - x1[0]) <= 1e-6 * np.linalg.norm(x1[0])
    assert np.linalg.norm(xm2[0] * 4.0 - xm1[0]) <= 1e-6 * np.linalg.norm(xm1[0])
