"""Runs the kernels of one workload a few times, for profilers (ncu).

    python profile_case.py --case c2 --reps 3 [--what matvec|cg|mixed]
        [--kernel staged --width 7] [--cg-form 0|2:smem|...]
    python profile_case.py --what batch --count 24 [--precision mixed|fp64]
    python profile_case.py --case c2 --what spmm|bcg|sample|restrict [--nrhs 8]
    python profile_case.py --what assemble

`matvec` runs the reference matvec demo's loop body (matvecmain.cpp:70-86):
L2GMap::update then Matrix::mult over all ranks, `reps` times, as plain
kernel launches.  `cg` runs one spmv::cg solve: a CUDA graph, or one
cooperative launch of the fused kernel (`--cg-form` forces the form through
SPMV_B200_CG_FUSED, so no timing launches precede the solve).  `mixed`
runs one mixed-precision solve to 1e-10 (`--cg-form` then forces its form
through SPMV_B200_CG_MIXED_FUSED).  `batch` runs one batched solve (one
cooperative launch) of the first `count` systems of the batched k-NN
workload with system 0's 32-column block, to 1e-10.  `spmm` runs
`reps` block products of `nrhs` right-hand sides (Matrix::operator* on a
block), `bcg` one block CG solve of `nrhs` columns to the workload's
tolerance, `sample` `reps` dL/dA samplings (-lambda_i x_j on the pattern),
`restrict` `reps` passes of transpmult + reverse_update (restrictmain.cpp's
loop body).  `assemble` runs one create_matrix on the device (Matrix.cpp:
213-438): the 5-point assembly of a 512^2 node grid over 8 ranks.
"""
from __future__ import annotations

import argparse

import numpy as np


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", default="c2")
    ap.add_argument("--scale", type=int, default=0)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--what", default="matvec",
                    choices=["matvec", "cg", "mixed", "batch", "spmm", "bcg", "sample",
                             "restrict", "assemble"])
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--count", type=int, default=24)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--kernel", default="auto", choices=["auto", "vector", "merge", "sell", "staged"])
    ap.add_argument("--width", type=int, default=0)
    ap.add_argument("--cg-form", default=None)
    args = ap.parse_args()
    if args.cg_form is not None:
        import os
        var = "SPMV_B200_CG_MIXED_FUSED" if args.what == "mixed" else "SPMV_B200_CG_FUSED"
        os.environ[var] = args.cg_form

    import torch
    import spmv_b200 as S
    from spmv_b200 import gen

    if args.what == "assemble":
        # One create_matrix on the device: the 5-point assembly of a 512^2
        # node grid over 8 ranks (repeated couplings summed, ghost rows routed
        # to their owners).
        nx, P = 512, 8
        bl, nrl, rgs, cgs = gen.grid_assembly_5pt(nx, P)
        M = S.create_matrix(S.Comm(size=P, device=0), bl, nrl, nrl, rgs, cgs)
        print("assemble", nx, "x", nx, "ranks", P, "entries in",
              sum(len(b[1]) for b in bl), "out", sum(M.nnz(q) for q in range(P)))
        return

    if args.what == "batch":
        from spmv_b200.core import Batch
        systems = gen.c4_systems(count=args.count)
        comm = S.Comm(size=1, device=0)
        B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in systems], block=(0, 32))
        bs = [torch.from_numpy(b).cuda() for _, b in systems]
        Bb = torch.from_numpy(gen.c4_block_rhs(systems[0][0].nrows)).cuda()
        x, info, X, binfo = B.solve(bs, 20000, 1e-10, block_b=Bb, precision=args.precision)
        print("batch", args.count, "systems", B.stats(), "config", B.config(args.precision),
              "converged", sum(i.converged for i in info) + sum(i.converged for i in binfo),
              "max iterations", max(i.iterations for i in info + binfo))
        return

    W = gen.workload(args.case, args.scale)
    D = gen.distribute(W.A, W.P)
    dt = np.float64 if args.dtype == "f64" else np.float32
    tdt = torch.float64 if args.dtype == "f64" else torch.float32
    comm = S.Comm(size=W.P, device=0)
    cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
    rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(W.P)])
    M = S.Matrix(comm, [(rp, ci, va.astype(dt)) for rp, ci, va in D.blocks], cm, rm)
    M.set_kernel(args.kernel, args.width)
    if args.what == "matvec":
        xs = [torch.rand(cm.vec_len(q), dtype=tdt, device="cuda") for q in range(W.P)]
        ys = [torch.empty(D.local_sizes[q], dtype=tdt, device="cuda") for q in range(W.P)]
        for _ in range(args.reps):
            cm.update(xs)
            M.mult(xs, out=ys)
        comm.synchronize()
        print("matvec", args.case, "reps", args.reps, "kernel", M.get_kernel())
    elif args.what == "mixed":
        b = [torch.from_numpy(W.b[D.ranges[q]:D.ranges[q + 1]].copy()).cuda()
             for q in range(W.P)]
        x, info = S.cg_mixed(comm, M, b, 20000, 1e-10)
        print("mixed", args.case, "inner iterations", info.iterations, "refinements",
              info.refinements, "form", M.cg_form("mixed"), "products",
              M.solver_product("mixed32"), M.solver_product("mixed64"))
    elif args.what == "spmm":
        X = [torch.rand((cm.vec_len(q), args.nrhs), dtype=tdt, device="cuda")
             for q in range(W.P)]
        for _ in range(args.reps):
            Y = M.mult_block(X)
        comm.synchronize()
        print("spmm", args.case, "nrhs", args.nrhs, "reps", args.reps)
    elif args.what == "bcg":
        Bm = [torch.rand((D.local_sizes[q], args.nrhs), dtype=torch.float64, device="cuda")
              for q in range(W.P)]
        from spmv_b200.core import cg_block
        X, infos = cg_block(comm, M, Bm, 10000, W.rtol)
        print("bcg", args.case, "nrhs", args.nrhs, "iterations", [i.iterations for i in infos])
    elif args.what == "sample":
        lam = [torch.rand(D.local_sizes[q], dtype=torch.float64, device="cuda")
               for q in range(W.P)]
        xs = [torch.rand(cm.vec_len(q), dtype=torch.float64, device="cuda") for q in range(W.P)]
        for _ in range(args.reps):
            out = M.sample_outer(lam, xs)
        comm.synchronize()
        print("sample", args.case, "reps", args.reps)
    elif args.what == "restrict":
        qs = [torch.rand(D.local_sizes[q], dtype=torch.float64, device="cuda")
              for q in range(W.P)]
        ps = [torch.empty(cm.vec_len(q), dtype=torch.float64, device="cuda") for q in range(W.P)]
        for _ in range(args.reps):
            M.transpmult(qs, out=ps)
            cm.reverse_update(ps)
        comm.synchronize()
        print("restrict", args.case, "reps", args.reps)
    else:
        b = [torch.from_numpy(W.b[D.ranges[q]:D.ranges[q + 1]].copy()).cuda()
             for q in range(W.P)]
        x, k = S.cg(comm, M, b, 10000, W.rtol)
        print("cg", args.case, "iterations", k, "form", M.cg_form(), "product",
              M.solver_product("cg"))


if __name__ == "__main__":
    main()
