"""Mixed-precision CG (FP32 inner iterations, FP64 refinement): converges to
the FP64 relative-residual target, confirmed in FP64, and its solution is
stated against the oracle's FP64 CG."""
import numpy as np
import pytest
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from helpers import build

pytestmark = pytest.mark.gpu


def solve_both(W, P, device=False):
    comm, cm, rm, M, D = build(W, P)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
    bb = [torch.from_numpy(v).cuda() for v in b] if device else b
    x, info = S.cg_mixed(comm, M, bb, 20000, W.rtol)
    if device:
        x = [v.cpu().numpy() for v in x]
    xm = np.concatenate([x[q][:D.local_sizes[q]] for q in range(P)])
    for q in range(P):
        assert np.all(x[q][D.local_sizes[q]:] == 0.0)
    x64, k64 = S.cg(comm, M, b, 20000, W.rtol)
    x64 = np.concatenate([x64[q][:D.local_sizes[q]] for q in range(P)])
    return xm, info, x64, k64, D


def relres(W, x):
    return np.linalg.norm(W.b - W.A.scipy() @ x) / np.linalg.norm(W.b)


@pytest.mark.parametrize("cfg,scale,P", [("c3", 24, 1), ("c2", 32, 8), ("c1", 64, 2)])
def test_mixed_reaches_fp64_target(cuda_device, cfg, scale, P):
    W = gen.workload(cfg, scale)
    W.rtol = 1e-10
    xm, info, x64, k64, D = solve_both(W, P, device=(cfg == "c2"))
    assert info.status == 0 and info.converged == 1
    assert info.relres < W.rtol
    assert relres(W, xm) < 1.5 * W.rtol          # independent FP64 check
    assert info.refinements >= 2
    # Inner iterations stay close to FP64 CG's (Krylov space carried over).
    assert info.iterations <= 1.5 * k64 + 20, (info.iterations, k64)
    # Error against the FP64 solution: bounded by the conditioning times the
    # residual target for both.
    err = np.linalg.norm(xm - x64) / np.linalg.norm(x64)
    assert err < 1e-6, err


def test_mixed_against_oracle_small(cuda_device):
    W = gen.workload("c3", 12)
    W.rtol = 1e-10
    xm, info, x64, k64, D = solve_both(W, 1)
    om = oracle.Map(D.local_sizes, D.ghosts)
    xo, ko, _ = oracle.cg(om, D.blocks, [W.b.copy()], 20000, 1e-10)
    err = np.linalg.norm(xm - xo[0]) / np.linalg.norm(xo[0])
    assert err < 1e-7, err


def test_mixed_zero_rhs_and_cap(cuda_device):
    W = gen.workload("c1", 32)
    comm, cm, rm, M, D = build(W, 1)
    x, info = S.cg_mixed(comm, M, [np.zeros(D.local_sizes[0])], 100, 1e-10)
    assert info.iterations == 0 and np.all(x[0] == 0)
    x, info = S.cg_mixed(comm, M, [W.b.copy()], 5, 1e-10)
    assert info.iterations == 5 and info.converged == 0
    # The capped solve still folded its correction into x (one refinement).
    assert info.refinements >= 1 and np.linalg.norm(x[0]) > 0
