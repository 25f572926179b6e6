"""Matrix::create_matrix (Matrix.cpp:213-438): assembly from rank blocks that
carry ghost rows, against the oracle's restatement (bitwise) and against the
global sum of the element matrices (scipy); host-only communicators, plus a
product and a solve on the GPU."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
import spmv_b200 as S


def fem_problem(nx, ny, P, dtype=np.float64, seed=0, spd=False):
    """Quad elements on an nx x ny node grid; element e goes to the rank that
    owns its lowest node.  Rank blocks list owned rows then ghost rows, with
    one entry per element contribution (repeats, element order)."""
    rng = np.random.default_rng(seed)
    n = nx * ny
    rr = S.owner_ranges(P, n)
    owner = lambda g: int(np.searchsorted(rr, g, side="right") - 1)  # noqa: E731
    contrib = [[] for _ in range(P)]   # (row, col, val) global
    glob = sp.lil_matrix((n, n), dtype=dtype)
    for j in range(ny - 1):
        for i in range(nx - 1):
            nodes = [j * nx + i, j * nx + i + 1, (j + 1) * nx + i, (j + 1) * nx + i + 1]
            if spd:
                K = np.array([[4, -1, -1, -2], [-1, 4, -2, -1], [-1, -2, 4, -1],
                              [-2, -1, -1, 4]], dtype=float) / 6.0 + np.eye(4) * 0.05
            else:
                K = rng.standard_normal((4, 4))
            if np.iscomplexobj(np.zeros(1, dtype)):
                K = K + 1j * rng.standard_normal((4, 4))
            K = K.astype(dtype)
            r = owner(min(nodes))
            for a in range(4):
                for b in range(4):
                    contrib[r].append((nodes[a], nodes[b], K[a, b]))
                    glob[nodes[a], nodes[b]] += K[a, b]
    blocks, nrl, ncl, rg, cg = [], [], [], [], []
    for r in range(P):
        r0, r1 = rr[r], rr[r + 1]
        rows = sorted({c[0] for c in contrib[r]} - set(range(r0, r1)))
        cols = sorted({c[1] for c in contrib[r]} - set(range(r0, r1)))
        rowlist = list(range(r0, r1)) + rows
        rpos = {g: k for k, g in enumerate(rowlist)}
        cpos = {g: (g - r0 if r0 <= g < r1 else (r1 - r0) + cols.index(g))
                for g in set(c[1] for c in contrib[r]) | set(range(r0, r1))}
        per = [[] for _ in rowlist]
        for (a, b, v) in contrib[r]:
            per[rpos[a]].append((cpos[b], v))
        rp = np.zeros(len(rowlist) + 1, np.int32)
        ci, va = [], []
        for k, lst in enumerate(per):
            for (c, v) in lst:
                ci.append(c)
                va.append(v)
            rp[k + 1] = len(ci)
        blocks.append((rp, np.array(ci, np.int32), np.array(va, dtype=dtype)))
        nrl.append(r1 - r0)
        ncl.append(r1 - r0)
        rg.append(np.array(rows, np.int64))
        cg.append(np.array(cols, np.int64))
    return blocks, nrl, ncl, rg, cg, sp.csr_matrix(glob), rr


@pytest.mark.parametrize("P", [1, 2, 3, 5])
@pytest.mark.parametrize("dtype", [np.float64, np.complex128])
def test_assembly_matches_oracle(P, dtype):
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(13, 11, P, dtype, seed=P)
    ref = oracle.create_matrix(blocks, nrl, ncl, rg, cg)
    comm = S.Comm(size=P, device=-1)
    M = S.create_matrix(comm, blocks, nrl, ncl, rg, cg)
    for r in range(P):
        rp, ci, va = M.mat(r)
        assert np.array_equal(rp, ref[r][0])
        assert np.array_equal(ci, ref[r][1])
        assert np.array_equal(va, ref[r][2].astype(dtype))
        assert np.array_equal(M.col_map().ghosts(r), ref[r][3])
        assert M.row_map().num_ghosts(r) == 0
        assert M.col_map().local_size(r) == ncl[r]


def test_oracle_assembly_is_the_global_sum():
    # Independent check of the restatement: mapped back to global columns,
    # the assembled rows are the element sum, rows in ascending column order.
    P = 4
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(17, 9, P, seed=11)
    ref = oracle.create_matrix(blocks, nrl, ncl, rg, cg)
    for r in range(P):
        rp, ci, va, gh = ref[r]
        glob = np.where(ci < ncl[r], ci + rr[r], gh[np.maximum(ci - ncl[r], 0)])
        B = sp.csr_matrix((va, glob, rp), shape=(nrl[r], G.shape[1]))
        assert abs(B - G[rr[r]:rr[r + 1]]).max() < 1e-12
        for i in range(nrl[r]):
            assert np.all(np.diff(ci[rp[i]:rp[i + 1]]) > 0)


def test_assembly_errors():
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(6, 5, 2, seed=3)
    comm = S.Comm(size=2, device=-1)
    bad = [g.copy() for g in rg]
    bad[1] = np.array([rr[1]] + list(bad[1][1:]), np.int64)  # a row rank 1 owns
    with pytest.raises(S.SpmvError, match="owned by its own rank"):
        S.create_matrix(comm, blocks, nrl, ncl, bad, cg)
    bad = [g.copy() for g in rg]
    bad[0] = bad[0].copy()
    bad[0][0] = 10**6
    with pytest.raises(S.SpmvError, match="out of range"):
        S.create_matrix(comm, blocks, nrl, ncl, bad, cg)


@pytest.mark.gpu
def test_assembled_product_and_solve(cuda_device):
    P = 3
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(40, 33, P, seed=5, spd=True)
    comm = S.Comm(size=P, device=0)
    M = S.create_matrix(comm, blocks, nrl, ncl, rg, cg)
    ref = oracle.create_matrix(blocks, nrl, ncl, rg, cg)
    cm = M.col_map()
    rng = np.random.default_rng(1)
    xg = rng.standard_normal(G.shape[1])
    xs = []
    for r in range(P):
        gh = cm.ghosts(r)
        xs.append(np.concatenate([xg[rr[r]:rr[r + 1]], xg[gh]]))
    ys = M.mult(xs)
    for r in range(P):
        yref = oracle.csr_mult(ref[r][0], ref[r][1], ref[r][2], xs[r])
        assert np.allclose(ys[r], yref, rtol=1e-12, atol=1e-14)
        assert np.allclose(ys[r], (G @ xg)[rr[r]:rr[r + 1]], rtol=1e-10, atol=1e-12)
    b = [rng.uniform(-1, 1, nrl[r]) for r in range(P)]
    x, k = S.cg(comm, M, b, 5000, 1e-10)
    om = oracle.Map(ncl, [ref[r][3] for r in range(P)])
    xo, ko, _ = oracle.cg(om, [(q[0], q[1], q[2]) for q in ref], b, 5000, 1e-10)
    assert abs(k - ko) <= 2
    for r in range(P):
        assert np.linalg.norm(x[r][:nrl[r]] - xo[r][:nrl[r]]) <= 1e-8 * np.linalg.norm(xo[r][:nrl[r]])


@pytest.mark.gpu
@pytest.mark.parametrize("P", [1, 2, 3, 5, 8])
@pytest.mark.parametrize("dtype", [np.float64, np.complex128, np.float32, np.complex64])
def test_device_assembly_matches_oracle(cuda_device, P, dtype):
    """The device assembly (routing, triplet sort, duplicate sums as kernels)
    is bitwise the oracle's restatement for FP64 types and the host assembly
    for all types."""
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(23, 19, P, dtype, seed=10 + P)
    M = S.create_matrix(S.Comm(size=P, device=0), blocks, nrl, ncl, rg, cg)
    H = S.create_matrix(S.Comm(size=P, device=-1), blocks, nrl, ncl, rg, cg)
    ref = (oracle.create_matrix(blocks, nrl, ncl, rg, cg)
           if dtype in (np.float64, np.complex128) else None)
    for r in range(P):
        rp, ci, va = M.mat(r)
        hp, hc, hv = H.mat(r)
        assert np.array_equal(rp, hp) and np.array_equal(ci, hc) and np.array_equal(va, hv)
        assert np.array_equal(M.col_map().ghosts(r), H.col_map().ghosts(r))
        if ref is not None:
            assert np.array_equal(rp, ref[r][0])
            assert np.array_equal(ci, ref[r][1])
            assert np.array_equal(va, ref[r][2].astype(dtype))
            assert np.array_equal(M.col_map().ghosts(r), ref[r][3])


@pytest.mark.gpu
def test_device_assembly_errors(cuda_device):
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(6, 5, 2, seed=3)
    comm = S.Comm(size=2, device=0)
    bad = [g.copy() for g in rg]
    bad[1] = np.array([rr[1]] + list(bad[1][1:]), np.int64)
    with pytest.raises(S.SpmvError, match="owned by its own rank"):
        S.create_matrix(comm, blocks, nrl, ncl, bad, cg)
    bcols = [(b[0], b[1].copy(), b[2]) for b in blocks]
    bcols[0][1][0] = 10**6       # a column outside the block
    with pytest.raises(S.SpmvError, match="column index outside the block"):
        S.create_matrix(comm, bcols, nrl, ncl, rg, cg)
    # An empty rank and a rank without ghost rows.
    P = 3
    blocks, nrl, ncl, rg, cg, G, rr = fem_problem(3, 2, P, seed=4)
    M = S.create_matrix(S.Comm(size=P, device=0), blocks, nrl, ncl, rg, cg)
    ref = oracle.create_matrix(blocks, nrl, ncl, rg, cg)
    for r in range(P):
        assert np.array_equal(M.mat(r)[2], ref[r][2])
