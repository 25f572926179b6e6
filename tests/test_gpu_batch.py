"""Batched solves: every system reaches ||b - A x|| / ||b|| < 1e-10 (checked
in FP64 here with scipy) in one persistent launch, for every cluster size,
and matches a direct FP64 solve."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import spmv_b200 as S
from spmv_b200 import gen
from spmv_b200.core import Batch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def systems():
    return gen.c4_systems(count=12, lo=300, hi=3000, seed=3)


@pytest.mark.parametrize("cluster", [1, 2, 4, 8])
def test_batch_converges_every_system(cuda_device, systems, cluster):
    comm = S.Comm(size=1, device=0)
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in systems], cluster=cluster)
    x, info = B.solve([b.copy() for _, b in systems], 20000, 1e-10)
    for (A, b), xi, inf in zip(systems, x, info):
        assert inf.status == 0 and inf.converged == 1, inf.iterations
        S_ = A.scipy()
        rel = np.linalg.norm(b - S_ @ xi) / np.linalg.norm(b)
        assert rel < 1.5e-10, rel
        xd = spla.spsolve(S_.tocsc(), b)
        assert np.linalg.norm(xi - xd) <= 1e-7 * np.linalg.norm(xd)


def test_batch_matches_single_mixed_solves(cuda_device, systems):
    comm = S.Comm(size=1, device=0)
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in systems])
    x, info = B.solve([b.copy() for _, b in systems], 20000, 1e-10)
    for (A, b), xi, inf in zip(systems[:4], x, info):
        cm = S.L2GMap(comm, [A.nrows], [[]])
        M = S.Matrix(comm, [(A.rowptr, A.cols, A.vals)], cm, cm)
        xm, im = S.cg_mixed(comm, M, [b.copy()], 20000, 1e-10)
        # Different FP32 summation orders take different paths; the counts
        # stay close and both solutions meet the same FP64 target.
        assert abs(inf.iterations - im.iterations) <= max(5, im.iterations // 4)
        assert np.linalg.norm(xi - xm[0]) <= 1e-8 * np.linalg.norm(xm[0])


def test_batch_device_vectors_and_edge_cases(cuda_device, systems):
    import torch
    comm = S.Comm(size=1, device=0)
    sub = systems[:3]
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in sub])
    bs = [torch.from_numpy(b.copy()).cuda() for _, b in sub]
    bs[1].zero_()                        # a zero right-hand side
    x, info = B.solve(bs, 20000, 1e-10)
    assert info[1].iterations == 0 and float(x[1].abs().max()) == 0.0
    assert info[0].converged == 1 and info[2].converged == 1
    x, info = B.solve(bs, 3, 1e-10)      # iteration cap
    assert info[0].iterations == 3 and info[0].converged == 0
