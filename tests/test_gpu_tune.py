"""The autotuner times candidate kernels on the matrix, keeps the fastest, and
the product and solvers stay correct with whatever it picks; its cache file
skips the timing for a matrix with the same statistics."""
import numpy as np
import pytest

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from helpers import TOL_F64, abs_mult, assert_spmv_close, build, random_csr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["c2", "random"])
def test_autotune_picks_a_working_kernel(cuda_device, case, tmp_path, monkeypatch):
    monkeypatch.setenv("SPMV_B200_TUNE_CACHE", str(tmp_path / "tune.txt"))
    if case == "c2":
        A = gen.workload("c2", 48).A
        P = 8
    else:
        A = random_csr(np.random.default_rng(0), 5000, 5000, density=0.003,
                       long_rows=(3,))
        P = 3
    comm, cm, rm, M, D = build(A, P)
    kernel, width, block, us, ncand = M.autotune(reps=5)
    assert ncand > 5 and us > 0
    assert M.get_kernel() == (kernel, width, block)
    rng = np.random.default_rng(1)
    xs = [rng.standard_normal(cm.vec_len(q)) for q in range(P)]
    ys = M.mult(xs)
    for q in range(P):
        rp, ci, va = D.blocks[q]
        assert_spmv_close(ys[q], oracle.csr_mult(rp, ci, va, xs[q]),
                          abs_mult(D.blocks[q], xs[q]), TOL_F64)
    # Same statistics: served from the cache.
    comm2, cm2, rm2, M2, D2 = build(A, P)
    k2 = M2.autotune(reps=5)
    assert k2[:3] == (kernel, width, block) and k2[4] == 0
    if case == "c2":
        W = gen.workload("c2", 48)
        b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
        x, k = S.cg(comm, M, b, 10000, W.rtol)
        xg = np.concatenate([x[q][:D.local_sizes[q]] for q in range(P)])
        rel = np.linalg.norm(W.b - W.A.scipy() @ xg) / np.linalg.norm(W.b)
        assert rel < 1.5 * W.rtol
