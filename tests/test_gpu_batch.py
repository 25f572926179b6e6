"""Batched solves (spmv_batch_solve_ex): k-NN graph Laplacians from the
batched workload's size range (4,096 .. 131,072 rows) and a 32-column block
of right-hand sides for one system, all in one cooperative launch.

Every system and every block column must reach ||b - A x|| / ||b|| < 1e-10,
checked here in FP64 with scipy, and agree with the oracle's FP64 CG
(cg.cpp:11-83 restated) run to 1e-12 (the solution error of a 1e-10
residual is bounded by cond(A) x 1e-10; cond(A) is about 1e2 for these
systems, so 1e-7 relative).  Small systems are also checked against scipy
direct solves."""
import os

import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen, _lib
from spmv_b200.core import Batch

pytestmark = pytest.mark.gpu

SIZES = [4096, 9000, 20011, 50000, 90001, 131072]
RTOL = 1e-10


def system(i, n):
    return gen.knn_laplacian(n, 12, 3, 1000 + i, 1e-2), gen.normal(3, 500 + i, n)


@pytest.fixture(scope="module")
def systems():
    return [system(i, n) for i, n in enumerate(SIZES)]


@pytest.fixture(scope="module")
def block_rhs():
    n = SIZES[-1]
    return np.stack([gen.normal(3, 700 + l, n) for l in range(32)], axis=1).copy()


def oracle_solve(A, b, rtol=1e-12):
    om = oracle.Map([A.nrows], [[]])
    x, k, _ = oracle.cg(om, [(A.rowptr, A.cols, A.vals)], [b], 20000, rtol, nthreads=8)
    return x[0], k


def relres(A, x, b):
    return np.linalg.norm(b - A.scipy() @ x) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def oracle_x(systems):
    return [oracle_solve(A, b) for A, b in systems]


def make_batch(systems, block=True):
    comm = S.Comm(size=1, device=0)
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in systems],
              block=(len(systems) - 1, 32) if block else None)
    return comm, B


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_with_block_against_oracle(cuda_device, systems, block_rhs, oracle_x, precision):
    comm, B = make_batch(systems)
    st = B.stats()
    assert st["rows"] == sum(SIZES) and st["index_bits"] == 16
    x, info, X, binfo = B.solve([b.copy() for _, b in systems], 20000, RTOL,
                                block_b=block_rhs.copy(), precision=precision)
    for i, ((A, b), xi, inf) in enumerate(zip(systems, x, info)):
        assert inf.status == 0 and inf.converged == 1, (i, inf.iterations)
        rr = relres(A, xi, b)
        assert rr < 1.5 * RTOL, (i, rr)
        assert abs(inf.relres - rr) <= 0.05 * rr + 1e-14, (i, inf.relres, rr)
        xo, ko = oracle_x[i]
        assert np.linalg.norm(xi - xo) <= 1e-7 * np.linalg.norm(xo), i
        if precision == "fp64":
            # Same recurrence on a renumbered system; the oracle ran to 1e-12,
            # so compare counts to a 1e-10 oracle run.
            _, k10 = oracle_solve(A, b, RTOL)
            assert abs(inf.iterations - k10) <= max(3, k10 // 50), (i, inf.iterations, k10)
    A, _ = systems[-1]
    for l, inf in enumerate(binfo):
        assert inf.status == 0 and inf.converged == 1, (l, inf.iterations)
        rr = relres(A, X[:, l], block_rhs[:, l])
        assert rr < 1.5 * RTOL, (l, rr)
    for l in (0, 13, 31):
        xo, _ = oracle_solve(A, block_rhs[:, l].copy())
        assert np.linalg.norm(X[:, l] - xo) <= 1e-7 * np.linalg.norm(xo), l


def test_batch_small_systems_against_direct_solves(cuda_device):
    sys_ = [system(10 + i, n) for i, n in enumerate([4096, 5000, 7777])]
    comm, B = make_batch(sys_, block=False)
    B.set_block(1, 5)
    Bb = np.stack([gen.normal(3, 900 + l, 5000) for l in range(5)], axis=1).copy()
    x, info, X, binfo = B.solve([b.copy() for _, b in sys_], 20000, RTOL, block_b=Bb)
    for (A, b), xi in zip(sys_, x):
        xd = spla.spsolve(A.scipy().tocsc(), b)
        assert np.linalg.norm(xi - xd) <= 1e-7 * np.linalg.norm(xd)
    A, _ = sys_[1]
    Xd = spla.spsolve(A.scipy().tocsc(), Bb)
    assert np.linalg.norm(X - Xd) <= 1e-7 * np.linalg.norm(Xd)
    assert all(i.converged == 1 for i in binfo)


def test_batch_launch_shapes_agree_and_repeat_bitwise(cuda_device, systems, block_rhs):
    sub = systems[:3] + [systems[-1]]
    comm, B = make_batch(sub)
    bs = [torch.from_numpy(b.copy()).cuda() for _, b in sub]
    Bd = torch.from_numpy(block_rhs.copy()).cuda()
    ref = None
    for cps, rows, lanes, win in [(2, 256, 32, True), (1, 128, 16, False), (2, 512, 16, False),
                                  (1, 256, 32, True)]:
        B.set_config(cps, rows, lanes, win)
        x, info, X, binfo = B.solve(bs, 20000, RTOL, block_b=Bd)
        xs = [v.cpu().numpy() for v in x]
        for (A, b), xi, inf in zip(sub, xs, info):
            assert inf.converged == 1 and relres(A, xi, b) < 1.5 * RTOL
        assert all(i.converged == 1 for i in binfo)
        if ref is None:
            ref = (xs, X.cpu().numpy())
        else:
            for a, c in zip(xs, ref[0]):
                assert np.linalg.norm(a - c) <= 1e-7 * np.linalg.norm(c)
        # The same shape twice: bitwise the same solve.
        x2, _, X2, _ = B.solve(bs, 20000, RTOL, block_b=Bd)
        for a, c in zip(x2, x):
            assert torch.equal(a, c)
        assert torch.equal(X2, X)


def test_batch_autotune_picks_a_resident_shape(cuda_device, systems, block_rhs):
    comm, B = make_batch(systems[:2] + [systems[-1]])
    for prec in ("mixed", "fp64"):
        cfg = B.autotune(prec)
        assert cfg["candidates"] >= 6 and cfg["us"] > 0
        assert cfg == {**B.config(prec), "us": cfg["us"], "candidates": cfg["candidates"]}
    x, info, X, binfo = B.solve([b.copy() for _, b in systems[:2] + [systems[-1]]], 20000,
                                RTOL, block_b=block_rhs.copy())
    assert all(i.converged == 1 for i in info) and all(i.converged == 1 for i in binfo)


def test_batch_matches_single_mixed_solves(cuda_device, systems):
    comm, B = make_batch(systems[:3], block=False)
    x, info = B.solve([b.copy() for _, b in systems[:3]], 20000, RTOL)
    for (A, b), xi, inf in zip(systems[:3], x, info):
        cm = S.L2GMap(comm, [A.nrows], [[]])
        M = S.Matrix(comm, [(A.rowptr, A.cols, A.vals)], cm, cm)
        xm, im = S.cg_mixed(comm, M, [b.copy()], 20000, RTOL)
        assert abs(inf.iterations - im.iterations) <= max(5, im.iterations // 4)
        assert np.linalg.norm(xi - xm[0]) <= 1e-8 * np.linalg.norm(xm[0])


def test_batch_edge_cases(cuda_device, systems):
    sub = [system(20 + i, n) for i, n in enumerate([300, 1000, 2000])]
    empty = gen.CSR(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), 0)
    comm = S.Comm(size=1, device=0)
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in sub] +
              [(empty.rowptr, empty.cols, empty.vals)])
    bs = [torch.from_numpy(b.copy()).cuda() for _, b in sub] + [torch.zeros(0, dtype=torch.float64,
                                                                            device="cuda")]
    bs[1].zero_()                        # a zero right-hand side
    x, info = B.solve(bs, 20000, RTOL)
    assert info[1].iterations == 0 and info[1].converged == 1
    assert float(x[1].abs().max()) == 0.0
    assert info[0].converged == 1 and info[2].converged == 1
    assert info[3].iterations == 0 and info[3].converged == 1
    x, info = B.solve(bs, 3, RTOL)       # iteration cap
    assert info[0].iterations == 3 and info[0].converged == 0
    assert info[0].refinements >= 1      # the cap confirms the residual in FP64
    x, info = B.solve(bs, 0, RTOL)       # no iterations at all
    assert info[0].iterations == 0 and float(x[0].abs().max()) == 0.0
    # Host vectors through the same entry point.
    xh, infoh = B.solve([b.copy() for _, b in sub] + [np.zeros(0)], 20000, RTOL)
    assert infoh[2].converged == 1 and relres(sub[2][0], xh[2], sub[2][1]) < 1.5 * RTOL


def test_batch_breakdown_is_reported(cuda_device):
    A, b = system(30, 500)
    Z = gen.CSR(A.rowptr.copy(), A.cols.copy(), np.zeros_like(A.vals), A.nrows)
    comm = S.Comm(size=1, device=0)
    B = Batch(comm, [(A.rowptr, A.cols, A.vals), (Z.rowptr, Z.cols, Z.vals)])
    with pytest.raises(S.SpmvError) as e:
        B.solve([b.copy(), b.copy()], 100, RTOL)
    assert e.value.status == _lib.ERROR_BREAKDOWN and "system 1" in str(e.value)


def test_batch_bounded_grid_wait(cuda_device, systems):
    # A limit of 1 ns makes the kernel's grid waits run out on a healthy
    # solve: the kernel returns, the host reports it, and the next solve on
    # the same batch succeeds.
    comm, B = make_batch(systems[:2], block=False)
    bs = [b.copy() for _, b in systems[:2]]
    os.environ["SPMV_B200_WAIT_LIMIT_NS"] = "1"
    try:
        with pytest.raises(S.SpmvError, match="timed out"):
            B.solve(bs, 20000, RTOL)
    finally:
        del os.environ["SPMV_B200_WAIT_LIMIT_NS"]
    x, info = B.solve(bs, 20000, RTOL)
    assert all(i.converged == 1 for i in info)


@pytest.mark.slow
def test_batch_full_workload(cuda_device):
    """The batched workload at full size: 256 systems of 4,096..131,072 rows
    and system 0's 32-column block, FP32 inner / FP64 refinement to 1e-10,
    one launch; every system and column confirmed in FP64 here."""
    systems = gen.c4_systems(count=256)
    n0 = systems[0][0].nrows
    Bb = gen.c4_block_rhs(n0)
    comm = S.Comm(size=1, device=0)
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in systems], block=(0, 32))
    bs = [torch.from_numpy(b).cuda() for _, b in systems]
    x, info, X, binfo = B.solve(bs, 20000, RTOL, block_b=torch.from_numpy(Bb).cuda())
    worst = 0.0
    for (A, b), xi, inf in zip(systems, x, info):
        assert inf.converged == 1 and inf.status == 0
        worst = max(worst, relres(A, xi.cpu().numpy(), b))
    Xh = X.cpu().numpy()
    for l in range(32):
        assert binfo[l].converged == 1
        worst = max(worst, relres(systems[0][0], Xh[:, l], Bb[:, l]))
    assert worst < 1.5 * RTOL, worst
