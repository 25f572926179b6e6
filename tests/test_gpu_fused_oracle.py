"""Every form of the CG solvers, forced one at a time, against the oracle's
restatement of spmv::cg (cg.cpp:11-83) at full size.

FP64 CG: the graph form and every fused plan (one, two or three CTAs per SM;
the residual in shared or global memory; three grid syncs per iteration, or
two in the merged-update form, ":m") on the 7-point 128^3 workload over
8 ranks (rtol 1e-8) and the 5-point 512^2 workload (rtol 1e-8): iterations
within 2 of the oracle's and x within 1e-9 (relative) of the oracle's x.

Mixed CG (FP32 inner iterations, FP64 refinement) to 1e-10: the graph form
and every fused plan on the 7-point workload, and the 27-point 160^3
lognormal workload in the form the library picks, against the oracle's FP64
CG run to 1e-10 on the same system.  Both meet ||b - A x|| / ||b|| < 1e-10,
so their difference is bounded by cond(A) x 2e-10; the tests state the
error they see and bound it at 1e-8."""
import numpy as np
import pytest

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from helpers import build

pytestmark = pytest.mark.gpu

CG_PLANS = ["0", "1:smem", "2:smem", "1:global", "2:global", "3:global", "2:smem:m", "3:global:m"]
MIXED_PLANS = ["0", "2:smem", "2:global", "3:global"]


def oracle_cg(W, D, rtol):
    om = oracle.Map(D.local_sizes, D.ghosts)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(D.P)]
    x, k, _ = oracle.cg(om, D.blocks, b, 20000, rtol, nthreads=oracle.max_threads())
    return np.concatenate([x[q][:D.local_sizes[q]] for q in range(D.P)]), k


@pytest.fixture(scope="module")
def c2():
    W = gen.workload("c2")
    D = gen.distribute(W.A, W.P)
    x8, k8 = oracle_cg(W, D, W.rtol)
    x10, k10 = oracle_cg(W, D, 1e-10)
    return W, {"1e-8": (x8, k8), "1e-10": (x10, k10)}


@pytest.fixture(scope="module")
def c1():
    W = gen.workload("c1")
    D = gen.distribute(W.A, W.P)
    return W, oracle_cg(W, D, W.rtol)


def gather(x, D):
    return np.concatenate([x[q][:D.local_sizes[q]].cpu().numpy()
                           if hasattr(x[q], "cpu") else x[q][:D.local_sizes[q]]
                           for q in range(D.P)])


def solve_fp64(monkeypatch, W, plan, width):
    monkeypatch.setenv("SPMV_B200_CG_FUSED", plan)
    comm, cm, rm, M, D = build(W, W.P)
    M.set_kernel("staged", width)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(W.P)]
    x, k = S.cg(comm, M, b, 20000, W.rtol)
    return gather(x, D), k, M


@pytest.mark.parametrize("plan", CG_PLANS)
def test_cg_form_against_oracle_c2(monkeypatch, cuda_device, c2, plan):
    W, ref = c2
    xo, ko = ref["1e-8"]
    x, k, M = solve_fp64(monkeypatch, W, plan, 7)
    form = M.cg_form()
    assert form[0] == ("graph" if plan == "0" else "fused")
    if plan != "0":
        assert (form[1], form[2]) == (int(plan[0]), plan[2:])
    assert abs(k - ko) <= 2, (k, ko)
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)


@pytest.mark.parametrize("plan", CG_PLANS)
def test_cg_form_against_oracle_c1(monkeypatch, cuda_device, c1, plan):
    W, (xo, ko) = c1
    x, k, M = solve_fp64(monkeypatch, W, plan, 5)
    assert M.cg_form()[0] == ("graph" if plan == "0" else "fused")
    assert abs(k - ko) <= 2, (k, ko)
    assert np.linalg.norm(x - xo) <= 1e-9 * np.linalg.norm(xo)


@pytest.mark.parametrize("plan", MIXED_PLANS)
def test_mixed_form_against_oracle_c2(monkeypatch, cuda_device, c2, plan):
    W, ref = c2
    xo, _ = ref["1e-10"]
    monkeypatch.setenv("SPMV_B200_CG_MIXED_FUSED", plan)
    comm, cm, rm, M, D = build(W, W.P)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(W.P)]
    x, info = S.cg_mixed(comm, M, b, 20000, 1e-10)
    assert M.cg_form("mixed")[0] == ("graph" if plan == "0" else "fused")
    assert info.converged == 1 and info.relres < 1e-10
    xg = gather(x, D)
    err = np.linalg.norm(xg - xo) / np.linalg.norm(xo)
    print("c2 mixed %s: %d inner iterations, %d refinements, error vs oracle %.2e"
          % (plan, info.iterations, info.refinements, err))
    assert err <= 1e-8, err
    rr = np.linalg.norm(W.b - W.A.scipy() @ xg) / np.linalg.norm(W.b)
    assert rr < 1.5e-10, rr


@pytest.mark.slow
def test_mixed_c3_full_size_against_oracle(cuda_device):
    """The 27-point lognormal 160^3 workload (4,096,000 rows) to 1e-10."""
    W = gen.workload("c3")
    D = gen.distribute(W.A, W.P)
    xo, ko = oracle_cg(W, D, 1e-10)
    comm, cm, rm, M, D = build(W, W.P)
    x, info = S.cg_mixed(comm, M, [W.b.copy()], 20000, 1e-10)
    assert info.converged == 1 and info.relres < 1e-10
    xg = gather(x, D)
    err = np.linalg.norm(xg - xo) / np.linalg.norm(xo)
    print("c3 mixed (%s): %d inner iterations, %d refinements (oracle FP64 CG: %d), "
          "error vs oracle %.2e" % (M.cg_form("mixed"), info.iterations, info.refinements,
                                    ko, err))
    assert err <= 1e-8, err
    rr = np.linalg.norm(W.b - W.A.scipy() @ xg) / np.linalg.norm(W.b)
    assert rr < 1.5e-10, rr
