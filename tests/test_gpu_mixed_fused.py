"""The fused mixed-precision CG solve (FP32 inner iterations with FP64
refinement as one cooperative launch of persistent CTAs) against its graph
form (three kernels per inner iteration, three more per refinement) on the
same matrix and staged products, for every fused plan: two CTAs per SM with
the FP32 residual in shared or global memory, or three with it in global
memory.  Also the edge cases through the fused form: zero right-hand side,
the iteration cap, ranks with no rows, run-to-run reproducibility and a grid
wait that runs out."""
import numpy as np
import pytest

import spmv_b200 as S
from spmv_b200 import gen
from helpers import build

pytestmark = pytest.mark.gpu

PLANS = ["2:smem", "2:global", "3:global"]


def solve(monkeypatch, plan, W, P, width, max_its=20000, rtol=1e-10):
    monkeypatch.setenv("SPMV_B200_CG_MIXED_FUSED", plan)
    comm, cm, rm, M, D = build(W, P)
    M.set_kernel("staged", width)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
    x, info = S.cg_mixed(comm, M, b, max_its, rtol)
    for q in range(P):
        assert np.all(x[q][D.local_sizes[q]:] == 0.0)
    xg = np.concatenate([x[q][:D.local_sizes[q]] for q in range(P)])
    return xg, info, M, comm, D


def true_relres(W, x):
    return np.linalg.norm(W.b - W.A.scipy() @ x) / np.linalg.norm(W.b)


@pytest.mark.parametrize("plan", PLANS)
@pytest.mark.parametrize("cfg,scale,P,width", [("c2", 32, 8, 8), ("c2", 40, 3, 4),
                                               ("c1", 64, 3, 5), ("c3", 24, 2, 9),
                                               ("c2", 32, 8, 7)])
def test_mixed_fused_matches_graph_form(monkeypatch, cuda_device, plan, cfg, scale, P, width):
    """Same per-element arithmetic as the graph form (FP32 products, FP64
    residual summed in storage order); only the grouping of the dot
    products' partial sums differs, so the iteration counts may differ by a
    few and the solutions agree to the residual target."""
    W = gen.workload(cfg, scale)
    rtol = 1e-10
    x0, i0, M0, _, _ = solve(monkeypatch, "0", W, P, width)
    assert M0.cg_form("mixed") == ("graph", 0, None)
    x1, i1, M1, _, _ = solve(monkeypatch, plan, W, P, width)
    cps, where = plan.split(":")
    assert M1.cg_form("mixed") == ("fused", int(cps), where)
    assert M1.solver_product("mixed32")[0] == "staged"
    assert i0.status == 0 and i1.status == 0
    assert i0.converged == 1 and i1.converged == 1
    assert i1.relres < rtol
    assert abs(i1.iterations - i0.iterations) <= max(3, i0.iterations // 20), (i0, i1)
    assert true_relres(W, x1) < 1.5 * rtol
    err = np.linalg.norm(x1 - x0) / np.linalg.norm(x0)
    assert err < 1e-6, err


@pytest.mark.parametrize("plan", PLANS)
def test_mixed_fused_zero_rhs_cap_and_repeat(monkeypatch, cuda_device, plan):
    W = gen.workload("c1", 32)
    monkeypatch.setenv("SPMV_B200_CG_MIXED_FUSED", plan)
    comm, cm, rm, M, D = build(W, 2)
    M.set_kernel("staged", 4)
    zero = [np.zeros(D.local_sizes[q]) for q in range(2)]
    x, info = S.cg_mixed(comm, M, zero, 100, 1e-10)
    assert M.cg_form("mixed")[0] == "fused"
    assert info.iterations == 0 and info.converged == 1
    assert all(np.all(v == 0) for v in x)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(2)]
    x, info = S.cg_mixed(comm, M, b, 5, 1e-10)
    assert info.iterations == 5 and info.converged == 0
    # The capped solve folded its correction into x (one refinement).
    assert info.refinements >= 1 and np.linalg.norm(np.concatenate(x)) > 0
    # Bitwise the same on a repeat (fixed reduction order).
    xa, ia = S.cg_mixed(comm, M, b, 20000, 1e-10)
    xb, ib = S.cg_mixed(comm, M, b, 20000, 1e-10)
    assert ia.iterations == ib.iterations and ia.refinements == ib.refinements
    assert all(np.array_equal(u, v) for u, v in zip(xa, xb))
    assert ia.converged == 1


@pytest.mark.parametrize("plan", PLANS)
def test_mixed_fused_empty_and_unaligned_ranks(monkeypatch, cuda_device, plan):
    """Ranks of 300, 0 and 724 rows (the last rank's rows start off the
    32-row slice grid; the middle rank owns nothing)."""
    W = gen.workload("c1", 32)
    monkeypatch.setattr(gen, "owner_ranges", lambda P, n: np.array([0, 300, 300, n]))
    out = {}
    for mode in ("0", plan):
        x, info, M, comm, D = solve(monkeypatch, mode, W, 3, 5)
        assert D.local_sizes == [300, 0, W.A.nrows - 300]
        assert M.cg_form("mixed")[0] == ("graph" if mode == "0" else "fused")
        assert info.status == 0 and info.converged == 1
        out[mode] = (x, info)
    (x0, i0), (x1, i1) = out["0"], out[plan]
    assert abs(i1.iterations - i0.iterations) <= 3
    assert np.linalg.norm(x1 - x0) <= 1e-6 * np.linalg.norm(x0)
    assert true_relres(W, x1) < 1.5e-10


def test_mixed_fused_wait_limit(monkeypatch, cuda_device):
    """A grid wait given 1 ns runs out: the kernel sets the error flag, every
    CTA leaves, and the host reports the timeout.  The context stays usable:
    the same matrix then solves with the default bound."""
    W = gen.workload("c2", 32)
    monkeypatch.setenv("SPMV_B200_CG_MIXED_FUSED", "2:smem")
    comm, cm, rm, M, D = build(W, 8)
    M.set_kernel("staged", 7)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(8)]
    monkeypatch.setenv("SPMV_B200_WAIT_LIMIT_NS", "1")
    with pytest.raises(S.SpmvError) as e:
        S.cg_mixed(comm, M, b, 20000, 1e-10)
    assert "timed out" in str(e.value)
    monkeypatch.delenv("SPMV_B200_WAIT_LIMIT_NS")
    x, info = S.cg_mixed(comm, M, b, 20000, 1e-10)
    assert M.cg_form("mixed")[0] == "fused" and info.converged == 1
    xg = np.concatenate([x[q][:D.local_sizes[q]] for q in range(8)])
    assert true_relres(W, xg) < 1.5e-10
