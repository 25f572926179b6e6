"""The seeded generators: the documented counter-based RNG, the sizes the
workloads are quoted at, symmetry, and the row-block distribution."""
import numpy as np
import pytest

from spmv_b200 import gen

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix(z):
    with np.errstate(over="ignore"):
        z = (z + np.uint64(0x9E3779B97F4A7C15))
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def np_uniform(seed, stream, n):
    with np.errstate(over="ignore"):
        k = _mix(_mix(np.uint64(seed)) ^ (np.uint64(stream) + np.uint64(0x632BE59BD9B4E019)))
        u = _mix(k + np.arange(n, dtype=np.uint64))
    return (u >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def test_uniform_matches_documented_formula():
    a = gen.uniform(7, 3, 1000, 0.0, 1.0)
    b = np_uniform(7, 3, 1000)
    assert np.array_equal(a, b)
    assert 0.0 <= a.min() and a.max() < 1.0


def test_normal_matches_box_muller():
    u = np_uniform(5, 9, 2000)
    ua, ub = u[0::2], u[1::2]
    rad = np.sqrt(-2.0 * np.log(1.0 - ua))
    z = np.empty(2000)
    z[0::2] = rad * np.cos(2 * np.pi * ub)
    z[1::2] = rad * np.sin(2 * np.pi * ub)
    assert np.allclose(gen.normal(5, 9, 2000), z, rtol=1e-14, atol=1e-14)


def _symmetric(A):
    S = A.scipy()
    return abs(S - S.T).max() == 0


def test_laplace_sizes():
    A = gen.laplace2d(512, 512)
    assert (A.nrows, A.nnz) == (262144, 1308672)
    A = gen.laplace3d(128)
    assert (A.nrows, A.nnz) == (2097152, 14581760)
    assert _symmetric(gen.laplace3d(8))


def test_27pt_structure():
    n = 12
    A = gen.laplace3d_27pt(n, 2, 1e-3)
    inner = (n - 2) ** 3
    assert A.nrows == n ** 3
    # 27*n^3 minus the missing neighbours of boundary layers.
    assert A.nnz == (3 * n - 2) ** 3
    assert _symmetric(A)
    S = A.scipy()
    rowsum = np.asarray(S.sum(axis=1)).ravel()
    assert np.allclose(rowsum, 1e-3, rtol=0, atol=1e-9)
    off = A.vals[A.vals < 0]
    # lognormal(0,1): median of -off near 1.
    assert 0.8 < np.median(-off) < 1.25
    assert inner > 0


def test_27pt_full_size_count():
    # 160^3 grid: (3n-2)^3 = 478^3 entries.
    assert (3 * 160 - 2) ** 3 == 109215352


def test_grid2d_softplus_edges():
    A = gen.grid2d_softplus(16, 16, 4, 0.5, 1e-3)
    ne = 2 * 16 * 15
    assert len(A.aux_f64) == ne and len(A.aux_i64) == 6 * ne
    edges = A.aux_i64[:2 * ne].reshape(ne, 2)
    pos = A.aux_i64[2 * ne:].reshape(ne, 4)
    w = np.log1p(np.exp(A.aux_f64))
    assert np.allclose(-A.vals[pos[:, 2]], w) and np.allclose(-A.vals[pos[:, 3]], w)
    assert np.array_equal(A.cols[pos[:, 2]], edges[:, 1])
    assert _symmetric(A)
    # 1024^2 quoted sizes
    assert 2 * 1024 * 1023 == 2095104 and 1024 * 1024 * 5 - 4 * 1024 == 5238784


def test_knn_graph():
    A = gen.knn_laplacian(5000, 12, 3, 0, 1e-2)
    assert A.nrows == 5000 and _symmetric(A)
    deg = np.diff(A.rowptr) - 1
    assert deg.min() >= 12 and 13 <= deg.mean() <= 20
    assert A.scalar > 0
    S = A.scipy()
    assert np.allclose(np.asarray(S.sum(axis=1)).ravel(), 1e-2, atol=1e-9)
    # k-NN exactness against brute force on a few points
    from spmv_b200.gen import uniform
    px, py, pz = (uniform(3, 10 * 0 + s, 5000, 0.0, 1.0) for s in (1, 2, 3))
    P = np.stack([px, py, pz], 1)
    for i in (0, 17, 4999):
        d = ((P - P[i]) ** 2).sum(1)
        d[i] = np.inf
        nn = set(np.argsort(d, kind="stable")[:12])
        row = set(A.cols[A.rowptr[i]:A.rowptr[i + 1]]) - {i}
        assert nn <= row


@pytest.mark.parametrize("P", [1, 2, 3, 8])
def test_distribute_reassembles(P):
    A = gen.laplace3d(10)
    D = gen.distribute(A, P)
    S = A.scipy().tocoo()
    rows, cols, vals = [], [], []
    for q in range(P):
        rp, ci, va = D.blocks[q]
        M = D.local_sizes[q]
        g = D.ghosts[q]
        assert np.all(np.diff(g) > 0)
        for i in range(M):
            seg = ci[rp[i]:rp[i + 1]]
            assert np.all(np.diff(seg) > 0)  # sorted by local column
            gpad = np.concatenate([g, [-1]])
            glob = np.where(seg < M, seg + D.ranges[q], gpad[np.maximum(seg - M, 0)])
            rows += [D.ranges[q] + i] * len(seg)
            cols += list(glob)
            vals += list(va[rp[i]:rp[i + 1]])
    import scipy.sparse as sp
    B = sp.coo_matrix((vals, (rows, cols)), shape=S.shape).tocsr()
    assert abs(B - A.scipy()).max() == 0
