"""spmv::cg on the GPU against the oracle's restatement of cg.cpp:11-83:
iteration counts within +-2, the same relative-residual target, matching
solutions, and the reference's error behaviour."""
import numpy as np
import pytest
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from helpers import GOLDEN, build

pytestmark = pytest.mark.gpu


def solve(W, P, device_vectors=False, max_its=10000):
    comm, cm, rm, M, D = build(W, P)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
    if device_vectors:
        bt = [torch.from_numpy(v).cuda() for v in b]
        x, k, info = S.cg(comm, M, bt, max_its, W.rtol, info=True)
        x = [v.cpu().numpy() for v in x]
    else:
        x, k, info = S.cg(comm, M, b, max_its, W.rtol, info=True)
    for q in range(P):
        assert x[q].shape == (cm.vec_len(q),)
        assert np.all(x[q][D.local_sizes[q]:] == 0.0)  # ghost tail zero
    xg = np.concatenate([x[q][:D.local_sizes[q]] for q in range(P)])
    return xg, k, info, D


def true_relres(W, x):
    return np.linalg.norm(W.b - W.A.scipy() @ x) / np.linalg.norm(W.b)


@pytest.mark.parametrize("key,cfg", [("c2_scale24_P8", "c2"), ("c1_scale64_P3", "c1")])
def test_small_cases_match_oracle(cuda_device, key, cfg):
    g = GOLDEN["cg"][key]
    W = gen.workload(cfg, g["scale"])
    x, k, info, D = solve(W, g["P"])
    om = oracle.Map(D.local_sizes, D.ghosts)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(g["P"])]
    xo, ko, _ = oracle.cg(om, D.blocks, b, 10000, W.rtol)
    assert ko == g["iterations"]  # the oracle still gives its pinned answer
    assert abs(k - ko) <= 2
    xog = np.concatenate([xo[q][:D.local_sizes[q]] for q in range(g["P"])])
    assert np.linalg.norm(x - xog) / np.linalg.norm(xog) < 1e-9
    assert true_relres(W, x) < 1.5 * W.rtol


@pytest.mark.parametrize("key,cfg", [("c1", "c1"), ("c2", "c2")])
def test_full_size_against_golden(cuda_device, key, cfg):
    g = GOLDEN["cg"][key]
    W = gen.workload(cfg)
    x, k, info, D = solve(W, g["P"], device_vectors=(cfg == "c2"))
    assert abs(k - g["iterations"]) <= 2, (k, g["iterations"])
    assert info.status == 0
    assert info.rnorm / info.rnorm0 < W.rtol ** 2
    assert true_relres(W, x) < 1.5 * W.rtol
    assert abs(x @ x - g["xnorm2"]) <= 1e-6 * g["xnorm2"]


def test_repeated_solves_are_reproducible(cuda_device):
    W = gen.workload("c2", 32)
    comm, cm, rm, M, D = build(W, 8)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(8)]
    x1, k1 = S.cg(comm, M, b, 10000, W.rtol)
    x2, k2 = S.cg(comm, M, b, 10000, W.rtol)
    assert k1 == k2 and all(np.array_equal(a, c) for a, c in zip(x1, x2))
    x3, k3 = S.cg(comm, M, b, 7, W.rtol)  # max_its caps the count
    assert k3 == 7


def test_zero_rhs(cuda_device):
    W = gen.workload("c1", 32)
    comm, cm, rm, M, D = build(W, 2)
    x, k = S.cg(comm, M, [np.zeros(n) for n in D.local_sizes], 100, 1e-8)
    assert k == 0 and all(np.all(v == 0) for v in x)


def test_negative_definite_converges(cuda_device):
    # CG does not need p.Ap > 0, only != 0: -A converges like A.
    W = gen.workload("c1", 48)
    neg = gen.CSR(W.A.rowptr, W.A.cols, -W.A.vals, W.A.ncols)
    Wn = gen.Workload("neg", neg, 1, W.b, W.rtol)
    x, k, info, D = solve(Wn, 2)
    xp, kp, _, _ = solve(W, 2)
    assert abs(k - kp) <= 2
    assert np.linalg.norm(x + xp) / np.linalg.norm(xp) < 1e-8


def test_breakdown_is_reported(cuda_device):
    W = gen.workload("c1", 16)
    zero = gen.CSR(W.A.rowptr, W.A.cols, 0.0 * W.A.vals, W.A.ncols)
    comm, cm, rm, M, D = build(zero, 1)
    with pytest.raises(S.SpmvError) as e:
        S.cg(comm, M, [W.b.copy()], 100, 1e-8)
    assert e.value.status == 5 and "breakdown" in str(e.value)


def test_reference_error_messages(cuda_device):
    W = gen.workload("c1", 16)
    comm, cm, rm, M, D = build(W, 2)
    with pytest.raises(S.SpmvError) as e:
        S.cg(comm, M, [np.zeros(3), np.zeros(D.local_sizes[1])], 10, 1e-8)
    assert str(e.value) == "spmv::cg - Error: b.rows() != A.rows()"
    # A row map with ghosts (cg.cpp:22-23).
    rg = S.L2GMap(comm, D.local_sizes, [[D.ranges[1]], []])
    blocks = [(np.concatenate([rp, [rp[-1]]]).astype(np.int32), ci, va)
              if q == 0 else (rp, ci, va) for q, (rp, ci, va) in enumerate(D.blocks)]
    M2 = S.Matrix(comm, blocks, cm, rg)
    with pytest.raises(S.SpmvError) as e:
        S.cg(comm, M2, [np.zeros(n) for n in D.local_sizes], 10, 1e-8)
    assert str(e.value) == "spmv::cg - Error: A.row_map() has ghost entries"


def test_matvec_demo_against_golden(cuda_device):
    """The reference's matvec demo (matvecmain.cpp:70-86): 1000 x {update;
    q = A psp; psp.head(M) = q} on create_A(500000), at 1 and 2 ranks."""
    N = 500000
    for P in (1, 2):
        A = gen.create_a(N)
        comm, cm, rm, M, D = build(A, P)
        psp = []
        for q in range(P):
            z = (np.arange(D.local_sizes[q]) + D.ranges[q]) / N
            v = np.zeros(cm.vec_len(q))
            v[:D.local_sizes[q]] = np.exp(-10 * (5 * (z - 0.5)) ** 2)
            psp.append(torch.from_numpy(v).cuda())
        qs = [torch.empty(D.local_sizes[q], dtype=torch.float64, device="cuda")
              for q in range(P)]
        stream = torch.cuda.ExternalStream(comm.stream)
        for _ in range(1000):
            cm.update(psp)
            M.mult(psp, out=qs)
            with torch.cuda.stream(stream):
                for q in range(P):
                    psp[q][:D.local_sizes[q]].copy_(qs[q])
        comm.synchronize()
        norm = sum(float((psp[q][:D.local_sizes[q]] ** 2).sum()) for q in range(P))
        ref = GOLDEN["matvec_demo_N500000_apply1000"][str(P)]
        assert abs(norm - ref) <= 1e-12 * ref, (P, norm, ref)


@pytest.mark.parametrize("cfg,scale,P,kernel,width", [
    ("c2", 32, 8, "sell", 8), ("c2", 32, 1, "vector", 4), ("c1", 64, 2, "vector", 2),
    ("c2", 32, 8, "staged", 8), ("c2", 40, 3, "staged", 4), ("c2", 32, 8, "auto", 0)])
def test_16bit_offsets_match_32bit_columns(cuda_device, monkeypatch, cfg, scale, P, kernel,
                                           width):
    """The solvers' 16-bit column offsets change only how indices are
    stored: with a vector or SELL product fixed, FP64 CG and mixed CG give
    bitwise the same answers with them on (default) and off (SPMV_B200_D16=0,
    read when the matrix's fused-halo columns are first built).  Otherwise
    (staged tiles, or the kernel left to the library's timing) the answers
    are compared to 1e-9 (FP64 CG) and 1e-6 (mixed)."""
    W = gen.workload(cfg, scale)
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("SPMV_B200_D16", flag)
        comm, cm, rm, M, D = build(W, P)
        M.set_kernel(kernel, width)
        b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
        x, k, _ = S.cg(comm, M, b, 10000, W.rtol, info=True)
        xm, im = S.cg_mixed(comm, M, b, 10000, W.rtol)
        assert im.converged
        for solver in ("cg", "mixed32", "mixed64"):
            kind, w, bits, us = M.solver_product(solver)
            assert us > 0 and bits in ((16, 32) if flag == "1" else (32,))
            if kernel != "auto":
                assert (kind, w) == (kernel, width)
        out[flag] = (x, k, xm, im.iterations)
    x1, k1, xm1, km1 = out["1"]
    x0, k0, xm0, km0 = out["0"]
    # Bitwise where the row-to-thread assignment does not depend on the index
    # width (vector, SELL); the staged tiles hold more 16-bit than 32-bit
    # entries, which changes the order of the dot products' partial sums.
    bitwise = kernel in ("vector", "sell")
    for q in range(P):
        if bitwise:
            assert k1 == k0 and km1 == km0
            assert np.array_equal(x1[q], x0[q])
            assert np.array_equal(xm1[q], xm0[q])
        else:
            assert abs(k1 - k0) <= 2
            assert np.linalg.norm(x1[q] - x0[q]) <= 1e-9 * np.linalg.norm(x0[q])
            assert np.linalg.norm(xm1[q] - xm0[q]) <= 1e-6 * np.linalg.norm(xm0[q])


def test_solver_product_needs_a_solve(cuda_device):
    W = gen.workload("c2", 16)
    comm, cm, rm, M, D = build(W, 2)
    with pytest.raises(S.SpmvError, match="has not run"):
        M.solver_product("cg")
    with pytest.raises(S.SpmvError, match="has not run"):
        M.solver_product("mixed32")


def test_solver_product_pin(cuda_device, monkeypatch):
    """SPMV_B200_SOLVER_PRODUCT keeps one product candidate (for profilers);
    a pin that names none of the matrix's candidates is refused."""
    W = gen.workload("c2", 24)
    monkeypatch.setenv("SPMV_B200_SOLVER_PRODUCT", "sell:4:32")
    comm, cm, rm, M, D = build(W, 2)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(2)]
    x, k = S.cg(comm, M, b, 10000, W.rtol)
    assert M.solver_product("cg")[:3] == ("sell", 4, 32)
    monkeypatch.setenv("SPMV_B200_SOLVER_PRODUCT", "sell:3:32")
    comm2, cm2, rm2, M2, D2 = build(W, 2)
    with pytest.raises(S.SpmvError) as e:
        S.cg(comm2, M2, b, 10000, W.rtol)
    assert "SPMV_B200_SOLVER_PRODUCT" in str(e.value)
