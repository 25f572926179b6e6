"""torch.autograd binding of the adjoint, used to check gradients.

`SpdSystem` holds one SPD matrix pattern on the GPU (one rank); `spd_solve`
is x = A(vals)^{-1} b as a torch.autograd.Function:

  forward:  x = cg(A(vals), b)
  backward: lambda = cg(A, dL/dx)           (A symmetric: A^T = A)
            dL/db    = lambda
            dL/dvals = -lambda_i x_j on A's pattern   (spmv_matrix_sample_outer)

Any parametrisation of vals (e.g. graph-Laplacian weights softplus(theta))
is ordinary torch code in front of it, so autograd carries dL/dvals on to
the parameters.
"""
from __future__ import annotations

import numpy as np
import torch

from . import core


class SpdSystem:
    def __init__(self, rowptr: np.ndarray, cols: np.ndarray, vals0: np.ndarray,
                 device: int = 0, rtol: float = 1e-12, max_its: int = 100000):
        n = len(rowptr) - 1
        self.n = n
        self.comm = core.Comm(size=1, device=device)
        self.cmap = core.L2GMap(self.comm, [n], [[]])
        self.rmap = core.L2GMap(self.comm, [n], [[]])
        self.M = core.Matrix(self.comm, [(rowptr, cols, np.asarray(vals0, np.float64))],
                             self.cmap, self.rmap)
        self.rtol = rtol
        self.max_its = max_its
        self.last_iterations = []

    def set_values(self, vals: torch.Tensor) -> None:
        self.M.set_values([vals.detach().to(torch.float64).contiguous()])

    def solve(self, b: torch.Tensor) -> torch.Tensor:
        b = b.detach().to(torch.float64).contiguous()
        x, k = core.cg(self.comm, self.M, [b], self.max_its, self.rtol)
        self.comm.synchronize()
        self.last_iterations.append(k)
        return x[0]


class _SpdSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vals, b, system):
        system.set_values(vals)
        x = system.solve(b)
        ctx.system = system
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        (x,) = ctx.saved_tensors
        system = ctx.system
        lam = system.solve(gx)
        gvals = system.M.sample_outer([lam], [x], -1.0)[0]
        system.comm.synchronize()
        return gvals, lam, None


def spd_solve(vals: torch.Tensor, b: torch.Tensor, system: SpdSystem) -> torch.Tensor:
    """x = A(vals)^{-1} b with gradients to vals and b."""
    return _SpdSolve.apply(vals, b, system)
