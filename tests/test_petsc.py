"""PETSc binary files (read_petsc.cpp): the library's reader against the
oracle's restatement and against the workload distribution, on host-only
communicators (no GPU), plus one solve from files on the GPU."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle
import spmv_b200 as S
from spmv_b200 import gen, petsc


def random_global(rng, nrows, ncols, density, shuffle=True, dup=False):
    """Global CSR with columns in random file order per row (optionally one
    repeated column in some rows)."""
    rp, ci, va = [0], [], []
    for i in range(nrows):
        k = int(rng.binomial(ncols, density))
        c = rng.choice(ncols, size=k, replace=False)
        if not shuffle:
            c = np.sort(c)
        if dup and k and rng.random() < 0.2:
            c = np.append(c, c[0])
        ci.extend(c.tolist())
        va.extend(rng.standard_normal(len(c)).tolist())
        rp.append(len(ci))
    return np.array(rp), np.array(ci, dtype=np.int64), np.array(va)


def blocks_of(M, P):
    return [M.mat(r) for r in range(P)]


@pytest.mark.parametrize("P", [1, 3, 8])
@pytest.mark.parametrize("shape", [(300, 300), (257, 190), (64, 500)])
def test_reader_matches_oracle(tmp_path, P, shape):
    rng = np.random.default_rng(P * 100 + shape[0])
    rp, ci, va = random_global(rng, *shape, density=0.03)
    f = tmp_path / "A.dat"
    petsc.write_matrix(f, rp, ci, va, shape[1])
    ref = oracle.petsc_read(f, P)
    comm = S.Comm(size=P, device=-1)
    M = S.read_petsc_binary(comm, f)
    cr = S.owner_ranges(P, shape[1])
    for r in range(P):
        rpo, cio, vao, gho = ref[r]
        rpl, cil, val = M.mat(r)
        assert np.array_equal(rpl, rpo)
        assert np.array_equal(cil, cio)
        assert np.array_equal(val, vao)
        cm = M.col_map()
        assert cm.local_size(r) == cr[r + 1] - cr[r]
        assert np.array_equal(cm.ghosts(r), gho)
        assert M.row_map().num_ghosts(r) == 0


def test_oracle_reader_against_scipy(tmp_path):
    # Independent check of the restatement: the blocks, mapped back to global
    # columns, are the file's matrix (repeated entries summed).
    rng = np.random.default_rng(7)
    n, m = 400, 350
    rp, ci, va = random_global(rng, n, m, density=0.02, dup=True)
    f = tmp_path / "A.dat"
    petsc.write_matrix(f, rp, ci, va, m)
    P = 4
    ref = oracle.petsc_read(f, P)
    rr, cr = S.owner_ranges(P, n), S.owner_ranges(P, m)
    A = sp.csr_matrix((va, ci, rp), shape=(n, m))
    for r in range(P):
        rpo, cio, vao, gho = ref[r]
        nloc = cr[r + 1] - cr[r]
        glob = np.where(cio < nloc, cio + cr[r], gho[np.maximum(cio - nloc, 0)])
        B = sp.csr_matrix((vao, glob, rpo), shape=(rr[r + 1] - rr[r], m))
        assert abs(B - A[rr[r]:rr[r + 1]]).max() < 1e-15
        # within a row, local columns ascend
        for i in range(len(rpo) - 1):
            assert np.all(np.diff(cio[rpo[i]:rpo[i + 1]]) >= 0)


def test_repeated_entries_keep_file_order(tmp_path):
    rng = np.random.default_rng(3)
    rp, ci, va = random_global(rng, 200, 200, density=0.05, dup=True)
    f = tmp_path / "A.dat"
    petsc.write_matrix(f, rp, ci, va, 200)
    ref = oracle.petsc_read(f, 2)
    M = S.read_petsc_binary(S.Comm(size=2, device=-1), f)
    for r in range(2):
        rpl, cil, val = M.mat(r)
        assert np.array_equal(cil, ref[r][1]) and np.array_equal(val, ref[r][2])


@pytest.mark.parametrize("cfg,P", [("c2", 8), ("c1", 3)])
def test_reader_gives_the_workload_blocks(tmp_path, cfg, P):
    # A square matrix with sorted rows read from a file is distributed exactly
    # as the workload generator distributes it (owner_ranges rows, owned
    # columns first, ghosts ascending).
    W = gen.workload(cfg, 24 if cfg == "c2" else 48)
    f = tmp_path / "A.dat"
    petsc.write_matrix(f, W.A.rowptr, W.A.cols, W.A.vals, W.A.ncols)
    D = gen.distribute(W.A, P)
    M = S.read_petsc_binary(S.Comm(size=P, device=-1), f)
    for r in range(P):
        rpl, cil, val = M.mat(r)
        rp, ci, va = D.blocks[r]
        assert np.array_equal(rpl, rp) and np.array_equal(cil, ci) and np.array_equal(val, va)
        assert np.array_equal(M.col_map().ghosts(r), D.ghosts[r])


@pytest.mark.parametrize("P", [1, 2, 5])
def test_vector_reader(tmp_path, P):
    v = np.random.default_rng(P).standard_normal(1001)
    f = tmp_path / "b.dat"
    petsc.write_vector(f, v)
    parts = S.read_petsc_binary_vector(S.Comm(size=P, device=-1), f)
    rr = S.owner_ranges(P, len(v))
    assert rr == list(oracle.owner_ranges(P, len(v)))
    for q in range(P):
        assert np.array_equal(parts[q], v[rr[q]:rr[q + 1]])


def test_reader_errors(tmp_path):
    comm = S.Comm(size=2, device=-1)
    with pytest.raises(S.SpmvError, match="Could not open file"):
        S.read_petsc_binary(comm, tmp_path / "missing.dat")
    with pytest.raises(S.SpmvError, match="Could not open file"):
        S.read_petsc_binary_vector(comm, tmp_path / "missing.dat")
    f = tmp_path / "v.dat"
    petsc.write_vector(f, np.ones(10))
    with pytest.raises(S.SpmvError, match="Bad signature in PETSc Matrix file"):
        S.read_petsc_binary(comm, f)
    g = tmp_path / "A.dat"
    petsc.write_matrix(g, [0, 1, 2], [0, 1], [1.0, 2.0], 2)
    with pytest.raises(S.SpmvError, match="Bad signature in PETSc Vector file"):
        S.read_petsc_binary_vector(comm, g)
    # truncated: drop the last value
    raw = g.read_bytes()
    t = tmp_path / "short.dat"
    t.write_bytes(raw[:-8])
    with pytest.raises(S.SpmvError, match="truncated"):
        S.read_petsc_binary(comm, t)
    # column index out of range
    bad = tmp_path / "bad.dat"
    petsc.write_matrix(bad, [0, 1, 2], [0, 5], [1.0, 2.0], 2)
    with pytest.raises(S.SpmvError, match="out of range"):
        S.read_petsc_binary(comm, bad)


@pytest.mark.gpu
def test_cg_from_petsc_files(tmp_path, cuda_device):
    # cgmain's flow (demos/cgmain.cpp): matrix and right-hand side from PETSc
    # files, then spmv::cg; compared with the oracle on the oracle's reading.
    W = gen.workload("c2", 24)
    fa, fb = tmp_path / "A.dat", tmp_path / "b.dat"
    petsc.write_matrix(fa, W.A.rowptr, W.A.cols, W.A.vals, W.A.ncols)
    petsc.write_vector(fb, W.b)
    P = 8
    comm = S.Comm(size=P, device=0)
    A = S.read_petsc_binary(comm, fa)
    b = S.read_petsc_binary_vector(comm, fb)
    x, k = S.cg(comm, A, b, 10000, W.rtol)
    ref = oracle.petsc_read(fa, P)
    om = oracle.Map([len(r[0]) - 1 for r in ref], [r[3] for r in ref])
    xo, ko, _ = oracle.cg(om, [(r[0], r[1], r[2]) for r in ref], b, 10000, W.rtol)
    assert abs(k - ko) <= 2
    for q in range(P):
        n = len(ref[q][0]) - 1
        assert np.linalg.norm(x[q][:n] - xo[q][:n]) <= 1e-9 * np.linalg.norm(xo[q][:n])
