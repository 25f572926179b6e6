"""The fused CG solve (spmv::cg, cg.cpp:11-83, as one cooperative launch of
persistent CTAs) against the graph form (three kernels per iteration) on the
same matrix and staged product, for every fused plan: one, two or three CTAs
per SM, the residual in shared or global memory, three grid syncs per
iteration or two (the merged-update form, ":m").  Also the reference's edge
cases through the fused form: zero right-hand side, the max_its cap,
breakdown, and run-to-run reproducibility."""
import numpy as np
import pytest

import spmv_b200 as S
from spmv_b200 import gen
from helpers import build

pytestmark = pytest.mark.gpu

PLANS = ["1:smem", "2:smem", "1:global", "2:global", "3:global", "2:smem:m", "3:global:m"]


def setup(monkeypatch, plan, W, P, width=8, kernel="staged"):
    monkeypatch.setenv("SPMV_B200_CG_FUSED", plan)
    comm, cm, rm, M, D = build(W, P)
    M.set_kernel(kernel, width)
    return comm, M, D


def solve(monkeypatch, plan, W, P, width=8, max_its=10000, kernel="staged"):
    comm, M, D = setup(monkeypatch, plan, W, P, width, kernel)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
    x, k, info = S.cg(comm, M, b, max_its, W.rtol, info=True)
    xg = np.concatenate([x[q][:D.local_sizes[q]] for q in range(P)])
    return xg, k, info, M


def true_relres(W, x):
    return np.linalg.norm(W.b - W.A.scipy() @ x) / np.linalg.norm(W.b)


@pytest.mark.parametrize("plan", PLANS)
@pytest.mark.parametrize("cfg,scale,P,width", [("c2", 32, 8, 8), ("c2", 40, 3, 4),
                                               ("c2", 32, 8, 7), ("c1", 64, 3, 5),
                                               ("c3", 24, 2, 9)])
def test_fused_matches_graph_form(monkeypatch, cuda_device, plan, cfg, scale, P, width):
    """Same per-element arithmetic as the graph form; the grouping of the
    dot products' partial sums differs, and the merged-update form takes
    beta from r.r - 2 alpha r.y + alpha^2 y.y (the next r.r in exact
    arithmetic)."""
    W = gen.workload(cfg, scale)
    x0, k0, i0, M0 = solve(monkeypatch, "0", W, P, width)
    assert M0.cg_form() == ("graph", 0, None)
    x1, k1, i1, M1 = solve(monkeypatch, plan, W, P, width)
    cps, where = plan.split(":", 1)
    assert M1.cg_form() == ("fused", int(cps), where)
    assert M1.solver_product("cg")[0] == "staged"
    assert i1.status == 0 and i0.status == 0
    assert abs(k1 - k0) <= 2, (k0, k1)
    assert np.linalg.norm(x1 - x0) <= 1e-9 * np.linalg.norm(x0)
    assert i1.rnorm / i1.rnorm0 < W.rtol ** 2
    assert true_relres(W, x1) < 1.5 * W.rtol


@pytest.mark.parametrize("plan", ["1:smem", "2:global", "2:smem:m"])
def test_fused_repeats_and_caps(monkeypatch, cuda_device, plan):
    W = gen.workload("c2", 32)
    comm, M, D = setup(monkeypatch, plan, W, 8)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(8)]
    x1, k1 = S.cg(comm, M, b, 10000, W.rtol)
    x2, k2 = S.cg(comm, M, b, 10000, W.rtol)
    assert M.cg_form()[0] == "fused"
    assert k1 == k2 and all(np.array_equal(a, c) for a, c in zip(x1, x2))
    x3, k3 = S.cg(comm, M, b, 7, W.rtol)  # max_its caps the count
    assert k3 == 7
    x4, k4 = S.cg(comm, M, [np.zeros(n) for n in D.local_sizes], 100, 1e-8)
    assert k4 == 0 and all(np.all(v == 0) for v in x4)
    # The workspace is reused after the zero right-hand side.
    x5, k5 = S.cg(comm, M, b, 10000, W.rtol)
    assert k5 == k1 and all(np.array_equal(a, c) for a, c in zip(x1, x5))


@pytest.mark.parametrize("plan", ["1:smem", "2:global", "2:smem:m"])
def test_fused_breakdown_is_reported(monkeypatch, cuda_device, plan):
    W = gen.workload("c1", 16)
    zero = gen.CSR(W.A.rowptr, W.A.cols, 0.0 * W.A.vals, W.A.ncols)
    monkeypatch.setenv("SPMV_B200_CG_FUSED", plan)
    comm, cm, rm, M, D = build(zero, 1)
    M.set_kernel("staged", 4)
    with pytest.raises(S.SpmvError) as e:
        S.cg(comm, M, [W.b.copy()], 100, 1e-8)
    assert e.value.status == 5 and "breakdown" in str(e.value)
    assert M.cg_form()[0] == "fused"


def test_fused_plan_that_does_not_fit_is_refused(monkeypatch, cuda_device):
    W = gen.workload("c2", 16)
    monkeypatch.setenv("SPMV_B200_CG_FUSED", "3:smem")
    comm, cm, rm, M, D = build(W, 2)
    M.set_kernel("staged", 8)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(2)]
    with pytest.raises(S.SpmvError):
        S.cg(comm, M, b, 100, W.rtol)


def test_staged_widths_accepted(cuda_device):
    """Staged widths are gathers in flight: 4, 5, 7, 8 or 9 (5, 7 and 9
    divide the 5-, 7- and 27-point stencils' rows); others are refused."""
    W = gen.workload("c2", 16)
    comm, cm, rm, M, D = build(W, 2)
    for w in (4, 5, 7, 8, 9):
        M.set_kernel("staged", w)
        assert M.get_kernel()[:2] == ("staged", w)
    with pytest.raises(S.SpmvError):
        M.set_kernel("staged", 6)
    with pytest.raises(S.SpmvError):
        M.set_kernel("sell", 7)


@pytest.mark.parametrize("plan", ["2:smem", "3:global", "2:smem:m"])
def test_fused_with_an_empty_rank_and_unaligned_ranks(monkeypatch, cuda_device, plan):
    """Ranks of 300, 0 and 724 rows (the last rank's rows start off the
    32-row slice grid; the middle rank owns nothing): the fused solve gives
    the graph form's answer."""
    W = gen.workload("c1", 32)
    monkeypatch.setattr(gen, "owner_ranges", lambda P, n: np.array([0, 300, 300, n]))
    out = {}
    for mode in ("0", plan):
        monkeypatch.setenv("SPMV_B200_CG_FUSED", mode)
        comm, cm, rm, M, D = build(W, 3)
        assert D.local_sizes == [300, 0, W.A.nrows - 300]
        M.set_kernel("staged", 5)
        b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(3)]
        x, k, info = S.cg(comm, M, b, 10000, W.rtol, info=True)
        assert info.status == 0 and M.cg_form()[0] == ("graph" if mode == "0" else "fused")
        assert x[1].size == 0
        out[mode] = (np.concatenate([x[q][:D.local_sizes[q]] for q in range(3)]), k)
    (x0, k0), (x1, k1) = out["0"], out[plan]
    assert abs(k1 - k0) <= 2
    assert np.linalg.norm(x1 - x0) <= 1e-9 * np.linalg.norm(x0)
    assert true_relres(W, x1) < 1.5 * W.rtol



@pytest.mark.parametrize("plan", ["2:smem", "3:global", "3:global:m"])
def test_fused_after_set_values(monkeypatch, cuda_device, plan):
    """New values on the same pattern reach the fused solve (its workspace
    keeps its plan and product).  Scaling A by 4 scales every product, alpha
    and x exactly in binary floating point, so the solve of 4A gives x/4 bit
    for bit in the same iterations."""
    W = gen.workload("c2", 32)
    monkeypatch.setenv("SPMV_B200_D16", "0")
    comm, M, D = setup(monkeypatch, plan, W, 8, 7)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(8)]
    x1, k1 = S.cg(comm, M, b, 10000, W.rtol)
    M.set_values([va * 4.0 for (rp, ci, va) in D.blocks])
    x2, k2 = S.cg(comm, M, b, 10000, W.rtol)
    assert M.cg_form()[0] == "fused"
    assert k2 == k1
    assert all(np.array_equal(a * 4.0, c) for a, c in zip(x2, x1))


def test_fused_wait_limit_reports_an_error(monkeypatch, cuda_device):
    """The fused solve's grid waits are bounded: with the bound at 1 ns every
    CTA that has to wait gives up at once, raises the device's error flag and
    leaves, and the host reports the timeout.  The context stays usable: the
    same matrix then solves with the default bound."""
    W = gen.workload("c2", 32)
    comm, M, D = setup(monkeypatch, "2:smem", W, 8, 7)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(8)]
    monkeypatch.setenv("SPMV_B200_WAIT_LIMIT_NS", "1")
    with pytest.raises(S.SpmvError) as e:
        S.cg(comm, M, b, 10000, W.rtol)
    assert "timed out" in str(e.value)
    monkeypatch.delenv("SPMV_B200_WAIT_LIMIT_NS")
    x, k, info = S.cg(comm, M, b, 10000, W.rtol, info=True)
    assert M.cg_form()[0] == "fused" and info.status == 0 and k > 0
    xg = np.concatenate([x[q][:D.local_sizes[q]] for q in range(8)])
    assert true_relres(W, xg) < 1.5 * W.rtol
