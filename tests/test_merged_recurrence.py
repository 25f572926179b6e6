"""The merged-update form of the fused CG (cg.cu cg_fused_solve_merged),
restated in numpy beside spmv::cg's recurrence (cg.cpp:11-83): the same
iterates and the same iteration count on small SPD systems.

The merged form takes beta from rr - 2 alpha r.y + alpha^2 y.y (the next
r.r in exact arithmetic, formed from the current true r.r) and tests the
true r.r of r_k one product later, before it would update x again; it stops
with x_k after k iterations, as cg.cpp does after its k-th update."""
import numpy as np
import pytest

from spmv_b200 import gen


def cg_reference(A, b, kmax, rtol):
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr0 = rr = r @ r
    k = 0
    while k < kmax:
        y = A @ p
        alpha = rr / (p @ y)
        x += alpha * p
        r -= alpha * y
        rr_new = r @ r
        k += 1
        if rr_new / rr0 < rtol * rtol:
            break
        p = p * (rr_new / rr) + r
        rr = rr_new
    return x, k


def cg_merged(A, b, kmax, rtol):
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = rr0 = r @ r
    k = 0
    while True:
        y = A @ p
        py, ry, yy = p @ y, r @ y, y @ y
        if (k > 0 and rr / rr0 < rtol * rtol) or k >= kmax:
            break
        alpha = rr / py
        beta = (rr - 2.0 * alpha * ry + alpha * alpha * yy) / rr
        r = r - alpha * y
        x = x + alpha * p
        p = p * beta + r
        rr = r @ r
        k += 1
    return x, k


@pytest.mark.parametrize("nx,rtol", [(24, 1e-8), (40, 1e-10)])
def test_merged_form_matches_cg(nx, rtol):
    A = gen.laplace2d(nx, nx).scipy().tocsr()
    b = gen.uniform(0, 0, A.shape[0])
    x0, k0 = cg_reference(A, b, 10000, rtol)
    x1, k1 = cg_merged(A, b, 10000, rtol)
    assert abs(k1 - k0) <= 1, (k0, k1)
    assert np.linalg.norm(x1 - x0) <= 1e-9 * np.linalg.norm(x0)
    assert np.linalg.norm(b - A @ x1) <= 1.01 * rtol * np.linalg.norm(b)


def test_merged_form_respects_the_cap():
    A = gen.laplace2d(16, 16).scipy().tocsr()
    b = gen.uniform(0, 0, A.shape[0])
    x0, k0 = cg_reference(A, b, 7, 1e-12)
    x1, k1 = cg_merged(A, b, 7, 1e-12)
    assert k0 == k1 == 7
    assert np.linalg.norm(x1 - x0) <= 1e-12 * np.linalg.norm(x0)
