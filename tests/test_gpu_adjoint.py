"""Adjoint of x = A(theta)^{-1} b: dL/dtheta and dL/db through
spmv_matrix_sample_outer + adjoint CG, bound to torch.autograd, checked
against an FP64 reference gradient (within 1e-6 relative) and against central
finite differences (eps = 1e-6, 64 random coordinates)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

import oracle
import spmv_b200 as S
from spmv_b200 import gen
from spmv_b200.autograd import SpdSystem, spd_solve
from helpers import build, random_csr

pytestmark = pytest.mark.gpu


def test_sample_outer_bitwise(cuda_device):
    rng = np.random.default_rng(3)
    A = random_csr(rng, 2000, 2000, density=0.004, long_rows=(11,))
    comm, cm, rm, M, D = build(A, 3)
    lam = [rng.standard_normal(D.local_sizes[q]) for q in range(3)]
    x = [rng.standard_normal(cm.vec_len(q)) for q in range(3)]
    for dev in (False, True):
        if dev:
            out = M.sample_outer([torch.from_numpy(v).cuda() for v in lam],
                                 [torch.from_numpy(v).cuda() for v in x])
            out = [o.cpu().numpy() for o in out]
        else:
            out = M.sample_outer(lam, x)
        for q in range(3):
            rp, ci, va = D.blocks[q]
            rows = np.repeat(np.arange(len(rp) - 1), np.diff(rp))
            assert np.array_equal(out[q], (-lam[q][rows]) * x[q][ci])


class GridProblem:
    """c5-style problem: A(theta) = L(softplus(theta)) + shift I on a grid."""

    def __init__(self, n, seed=4, shift=1e-3):
        self.G = gen.grid2d_softplus(n, n, seed, 0.5, shift)
        self.shift = shift
        ne = len(self.G.aux_f64)
        self.theta = self.G.aux_f64.copy()
        self.edges = self.G.aux_i64[:2 * ne].reshape(ne, 2)
        self.pos = self.G.aux_i64[2 * ne:].reshape(ne, 4)
        N = self.G.nrows
        self.b = gen.normal(seed, 100, N)
        self.xstar = gen.normal(seed, 101, N)
        self.diag = np.array([self.G.rowptr[i] + np.searchsorted(
            self.G.cols[self.G.rowptr[i]:self.G.rowptr[i + 1]], i) for i in range(N)])

    def vals_np(self, theta):
        w = np.logaddexp(0.0, theta)
        v = np.zeros(self.G.nnz)
        v[self.diag] = self.shift
        np.add.at(v, self.pos[:, 0], w)
        np.add.at(v, self.pos[:, 1], w)
        v[self.pos[:, 2]] = -w
        v[self.pos[:, 3]] = -w
        return v

    def vals_torch(self, theta_t):
        w = torch.nn.functional.softplus(theta_t)
        v = torch.zeros(self.G.nnz, dtype=torch.float64, device=theta_t.device)
        dev = theta_t.device
        v[torch.from_numpy(self.diag).to(dev)] = self.shift
        p = torch.from_numpy(self.pos).to(dev)
        v = v.index_add(0, p[:, 0], w).index_add(0, p[:, 1], w)
        v = v.index_add(0, p[:, 2], -w).index_add(0, p[:, 3], -w)
        return v

    def scipy_A(self, theta):
        return sp.csr_matrix((self.vals_np(theta), self.G.cols, self.G.rowptr),
                             shape=(self.G.nrows, self.G.nrows))

    def loss_direct(self, theta):
        x = spla.spsolve(self.scipy_A(theta).tocsc(), self.b)
        return 0.5 * np.sum((x - self.xstar) ** 2)

    def reference_grad(self, theta, solve):
        x = solve(theta, self.b)
        lam = solve(theta, x - self.xstar)
        i, j = self.edges[:, 0], self.edges[:, 1]
        sig = 1.0 / (1.0 + np.exp(-theta))
        return -(lam[i] - lam[j]) * (x[i] - x[j]) * sig, lam


def adjoint_grad(P: GridProblem, rtol):
    sysm = SpdSystem(P.G.rowptr, P.G.cols, P.vals_np(P.theta), rtol=rtol)
    th = torch.from_numpy(P.theta.copy()).cuda().requires_grad_(True)
    b = torch.from_numpy(P.b.copy()).cuda().requires_grad_(True)
    xs = torch.from_numpy(P.xstar).cuda()
    x = spd_solve(P.vals_torch(th), b, sysm)
    L = 0.5 * ((x - xs) ** 2).sum()
    L.backward()
    return th.grad.cpu().numpy(), b.grad.cpu().numpy(), float(L.detach()), sysm


def test_adjoint_small_grid_against_direct_fp64(cuda_device):
    P = GridProblem(40)
    g, gb, L, _ = adjoint_grad(P, 1e-13)

    def direct(theta, rhs):
        return spla.spsolve(P.scipy_A(theta).tocsc(), rhs)

    gref, lam = P.reference_grad(P.theta, direct)
    assert np.linalg.norm(g - gref) <= 1e-6 * np.linalg.norm(gref)
    assert np.linalg.norm(gb - lam) <= 1e-6 * np.linalg.norm(lam)
    assert abs(L - P.loss_direct(P.theta)) <= 1e-9 * L
    # Central finite differences on 64 random coordinates (direct FP64 solves).
    rng = np.random.default_rng(0)
    idx = rng.choice(len(P.theta), size=64, replace=False)
    eps = 1e-6
    fd = np.empty(64)
    for t, e in enumerate(idx):
        tp, tm = P.theta.copy(), P.theta.copy()
        tp[e] += eps
        tm[e] -= eps
        fd[t] = (P.loss_direct(tp) - P.loss_direct(tm)) / (2 * eps)
    # Central differences carry O(eps^2) truncation and the rounding of the
    # two losses divided by 2 eps; the exact FP64 gradient shows how large
    # that noise is here, and ours must agree with FD as well as it does.
    fd_noise = np.linalg.norm(fd - gref[idx])
    assert np.linalg.norm(fd - g[idx]) <= 1.5 * fd_noise + 1e-9 * np.linalg.norm(g[idx])
    assert np.linalg.norm(fd - g[idx]) <= 1e-4 * np.linalg.norm(g[idx])


def test_adjoint_full_size_c5(cuda_device):
    """1024^2 grid (2,095,104 theta): adjoint gradient within 1e-6 of the FP64
    reference gradient (oracle CG to 1e-13 on the host), and consistent with
    central differences on 64 coordinates (GPU solves at 1e-14)."""
    P = GridProblem(1024)
    g, gb, L, sysm = adjoint_grad(P, 1e-12)
    assert len(g) == 2095104

    om = oracle.Map([P.G.nrows], [np.zeros(0, np.int64)])
    nth = oracle.max_threads()

    def oracle_solve(theta, rhs):
        blk = [(P.G.rowptr, P.G.cols, P.vals_np(theta))]
        xs, k, _ = oracle.cg(om, blk, [rhs.copy()], 100000, 1e-13, nthreads=nth)
        return xs[0]

    gref, lam = P.reference_grad(P.theta, oracle_solve)
    rel = np.linalg.norm(g - gref) / np.linalg.norm(gref)
    assert rel <= 1e-6, rel
    assert np.linalg.norm(gb - lam) <= 1e-6 * np.linalg.norm(lam)

    rng = np.random.default_rng(1)
    idx = rng.choice(len(P.theta), size=64, replace=False)
    eps = 1e-6
    tight = SpdSystem(P.G.rowptr, P.G.cols, P.vals_np(P.theta), rtol=1e-14,
                      max_its=200000)
    xs = torch.from_numpy(P.xstar).cuda()
    bt = torch.from_numpy(P.b).cuda()

    def loss(theta):
        tight.set_values(torch.from_numpy(P.vals_np(theta)).cuda())
        x = tight.solve(bt)
        return float(0.5 * ((x - xs) ** 2).sum())

    fd = np.empty(64)
    for t, e in enumerate(idx):
        tp, tm = P.theta.copy(), P.theta.copy()
        tp[e] += eps
        tm[e] -= eps
        fd[t] = (loss(tp) - loss(tm)) / (2 * eps)
    fd_noise = np.linalg.norm(fd - gref[idx])
    err = np.linalg.norm(fd - g[idx])
    assert err <= 1.5 * fd_noise + 1e-9 * np.linalg.norm(g[idx]), (err, fd_noise)
    assert err <= 1e-3 * np.linalg.norm(g[idx]), err
