"""Benchmark of the spmv_b200 hot path (one JSON line on rank 0).

Workload (default): 3D 7-point Laplacian on 128^3 (2,097,152 rows,
14,581,760 nnz), FP64 CSR with int32 indices, split into 8 row-block ranks with
L2GMap ghosts on one GPU; b ~ U[-1,1] (seed 1); x0 = 0.

A step is one FP64 CG solve to relative residual 1e-8 through spmv::cg's
device path (b and x device-resident).  `value` = solves/s over the whole job.
`e2e` is the same solve through the C ABI with pinned host b and x (the
host->device copy of b and device->host copy of x inside the timed region).
`roofline` covers the kernel that runs the timed steps: with the fused solve
(one cooperative launch per solve) that kernel, its duration the step time
measured with CUDA events on the library's stream, its algorithmic bytes
B_iter x iterations (B_iter: the product's bytes plus 9 n vector terms);
with the graph form, the CSR product.  `mult_roofline` always covers the CSR
product, timed live over repeated launches of Matrix::mult.

`--impl reference` times the reference's CPU path instead: the oracle's
restatement of spmv::cg (Eigen/MKL/MPI are not available to build the real
reference) on all host threads, one complete solve per step.

Multi-GPU (torchrun, N > 1): replicas only.  Each rank solves its own copy of
the workload on its own GPU (no data-path collective); `value` sums solves over
ranks divided by the max-over-ranks time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "c2"
MEASURED_PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 2 ** 20


def peaks():
    try:
        d = json.loads(MEASURED_PEAKS.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# Clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) != 6:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


# ---------------------------------------------------------------------------
# Workload
# ---------------------------------------------------------------------------
def spmv_bytes(n, nnz, P, g, sv=8, si=4):
    """Algorithmic bytes of one update + SpMV (values+cols, rowptr per rank,
    x owned+ghost read once, y written once, ghost gather)."""
    return nnz * (sv + si) + (n + P) * si + (n + g) * sv + n * sv + g * (2 * sv + si)


def kernel_bytes(n, nnz, P, g, sv=8, si=4):
    """Algorithmic bytes of the product kernel alone (no ghost gather)."""
    return nnz * (sv + si) + (n + P) * si + (n + g) * sv + n * sv


def setup(device: int):
    import spmv_b200 as S
    from spmv_b200 import gen
    W = gen.workload(WORKLOAD)
    D = gen.distribute(W.A, W.P)
    comm = S.Comm(size=W.P, device=device)
    cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
    rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(W.P)])
    M = S.Matrix(comm, D.blocks, cm, rm)
    M.autotune(reps=10)  # the plan step: pick kernel, width and block
    return W, D, comm, cm, rm, M


def dist_init():
    from spmv_b200 import ranks
    info = ranks.init("nccl")
    return info


def max_over_ranks(v: float, info) -> float:
    from spmv_b200 import ranks
    return ranks.max_over_ranks(v, info)


def barrier(info):
    from spmv_b200 import ranks
    ranks.barrier(info)


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_full_solve(W, D, nthreads: int):
    """One complete oracle spmv::cg solve (cg.cpp:11-83 restated) on
    `nthreads` host threads; returns (seconds, iterations)."""
    import oracle
    om = oracle.Map(D.local_sizes, D.ghosts)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(D.P)]
    t0 = time.perf_counter()
    _, k, _ = oracle.cg(om, D.blocks, b, 10000, W.rtol, nthreads=nthreads)
    return time.perf_counter() - t0, k


def cpu_sample(W, D, budget_s: float, nthreads: int):
    """Times the oracle's spmv::cg for a bounded number of iterations (about
    budget_s seconds); returns (seconds per iteration, iterations run)."""
    import oracle
    om = oracle.Map(D.local_sizes, D.ghosts)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(D.P)]
    t0 = time.perf_counter()
    oracle.cg(om, D.blocks, b, 10000, W.rtol, nthreads=nthreads, max_its_run=3)
    per = (time.perf_counter() - t0) / 3
    its = int(max(3, min(2000, budget_s / max(per, 1e-6))))
    t0 = time.perf_counter()
    _, k, _ = oracle.cg(om, D.blocks, b, 10000, W.rtol, nthreads=nthreads,
                        max_its_run=its)
    dt = time.perf_counter() - t0
    return dt / k, k


def config_dict(W, D, P, extra=None):
    g = int(sum(len(x) for x in D.ghosts))
    c = {"workload": "3D 7-point Laplacian 128^3 (c2): n=2097152, nnz=14581760, "
                     "8 row-block ranks on one GPU, ghosts=%d; FP64 CG to rel-res 1e-8, "
                     "b~U[-1,1] seed 1" % g,
         "n": W.A.nrows, "nnz": W.A.nnz, "ranks": P, "ghosts": g, "rtol": W.rtol,
         "l2": "working set (matrix 223 MB + CG vectors) exceeds the 126 MB L2; "
               "no flush between steps",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# Mixed-precision and batched solves against plain FP64 GPU CG (rel-res 1e-10)
# ---------------------------------------------------------------------------
def _timed(stream, fn, reps):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps, out


def run_extras(device: int, reps: int, c4_count: int, which=("c3", "c2", "c4", "c5", "next")):
    """c3: 27-point lognormal Laplacian 160^3 (4,096,000 rows), FP64 CG vs
    mixed CG, both to ||b - A x|| / ||b|| < 1e-10; c2: the same on the
    7-point 128^3 Poisson matrix over 8 ranks (the CG workload); c4: the
    batched workload (run_c4); c5: one adjoint (forward solve, adjoint solve,
    dL/dA sampling) on the 1024^2 grid; next: the rows beyond the CG path.
    `which` selects the parts."""
    import torch
    import spmv_b200 as S
    from spmv_b200 import gen
    from spmv_b200.core import Batch
    out = {}
    if "c3" in which:
        t0 = time.perf_counter()
        W = gen.workload("c3")
        comm = S.Comm(size=1, device=device)
        stream = comm.torch_stream()
        cm = S.L2GMap(comm, [W.A.nrows], [[]])
        M = S.Matrix(comm, [(W.A.rowptr, W.A.cols, W.A.vals)], cm, cm)
        tune = M.autotune(reps=5)
        b = [torch.from_numpy(W.b).cuda(device)]
        x64 = [torch.zeros_like(b[0])]
        xm = [torch.zeros_like(b[0])]
        _, k64 = S.cg(comm, M, b, 20000, 1e-10, x=x64)
        _, im = S.cg_mixed(comm, M, b, 20000, 1e-10, x=xm)
        setup_s = time.perf_counter() - t0
        t64, (_, k64) = _timed(stream, lambda: S.cg(comm, M, b, 20000, 1e-10, x=x64), reps)
        tmx, (_, im) = _timed(stream, lambda: S.cg_mixed(comm, M, b, 20000, 1e-10, x=xm), reps)
        r = M.mult(xm)[0]
        relres_m = float(torch.linalg.norm(b[0] - r) / torch.linalg.norm(b[0]))
        r = M.mult(x64)[0]
        relres_64 = float(torch.linalg.norm(b[0] - r) / torch.linalg.norm(b[0]))
        err = float(torch.linalg.norm(xm[0] - x64[0]) / torch.linalg.norm(x64[0]))
        out["c3_mixed_vs_fp64"] = {
            "fp64_cg_solves_per_s": 1.0 / t64, "fp64_iterations": k64,
            "mixed_solves_per_s": 1.0 / tmx, "mixed_inner_iterations": im.iterations,
            "mixed_refinements": im.refinements, "speedup": t64 / tmx,
            "relres_fp64": relres_64, "relres_mixed": relres_m,
            "error_mixed_vs_fp64_solution": err, "mult_kernel": tune[:3],
            "cg_product": M.solver_product("cg"),
            "mixed_products": [M.solver_product("mixed32"), M.solver_product("mixed64")],
            "cg_form": M.cg_form(), "mixed_form": M.cg_form("mixed"),
            "setup_s": setup_s}
        del M, cm, b, x64, xm
        torch.cuda.empty_cache()
    if "c2" in which:
        W = gen.workload("c2")
        D = gen.distribute(W.A, W.P)
        comm2 = S.Comm(size=W.P, device=device)
        stream2 = comm2.torch_stream()
        cm = S.L2GMap(comm2, D.local_sizes, D.ghosts)
        rm = S.L2GMap(comm2, D.local_sizes, [[] for _ in range(W.P)])
        M = S.Matrix(comm2, D.blocks, cm, rm)
        b = [torch.from_numpy(W.b[D.ranges[q]:D.ranges[q + 1]].copy()).cuda(device)
             for q in range(W.P)]
        x64 = [torch.zeros(cm.vec_len(q), dtype=torch.float64, device=f"cuda:{device}")
               for q in range(W.P)]
        xm = [torch.zeros_like(v) for v in x64]
        S.cg(comm2, M, b, 20000, 1e-10, x=x64)
        S.cg_mixed(comm2, M, b, 20000, 1e-10, x=xm)
        t64, (_, k64) = _timed(stream2, lambda: S.cg(comm2, M, b, 20000, 1e-10, x=x64), reps)
        tmx, (_, im) = _timed(stream2, lambda: S.cg_mixed(comm2, M, b, 20000, 1e-10, x=xm), reps)
        xa = torch.cat([xm[q][:D.local_sizes[q]] for q in range(W.P)])
        xb = torch.cat([x64[q][:D.local_sizes[q]] for q in range(W.P)])
        out["c2_mixed_vs_fp64"] = {
            "fp64_cg_solves_per_s": 1.0 / t64, "fp64_iterations": k64,
            "mixed_solves_per_s": 1.0 / tmx, "mixed_inner_iterations": im.iterations,
            "mixed_refinements": im.refinements, "speedup": t64 / tmx,
            "relres_mixed": im.relres,
            "error_mixed_vs_fp64_solution": float(torch.linalg.norm(xa - xb) /
                                                  torch.linalg.norm(xb)),
            "cg_form": M.cg_form(), "mixed_form": M.cg_form("mixed"),
            "mixed_products": [M.solver_product("mixed32"), M.solver_product("mixed64")]}
        del M, cm, rm, b, x64, xm
        torch.cuda.empty_cache()
    if "c4" in which:
        out["c4_batched"] = run_c4(device, reps)
        torch.cuda.empty_cache()
    if "c5" in which:
        from spmv_b200.autograd import SpdSystem, spd_solve
        G = gen.grid2d_softplus(1024, 1024, 4, 0.5, 1e-3)
        sysm = SpdSystem(G.rowptr, G.cols, G.vals, device=device, rtol=1e-12)
        bt = torch.from_numpy(gen.normal(4, 100, G.nrows)).cuda(device)
        xs = torch.from_numpy(gen.normal(4, 101, G.nrows)).cuda(device)
        vals = torch.from_numpy(G.vals).cuda(device).requires_grad_(True)

        def adjoint():
            vals.grad = None
            x = spd_solve(vals, bt, sysm)
            L = 0.5 * ((x - xs) ** 2).sum()
            L.backward()
            return L

        adjoint()
        ta, _ = _timed(torch.cuda.current_stream(device), adjoint, 1)
        out["c5_adjoint"] = {"forward_plus_adjoint_s": ta,
                             "cg_iterations": sysm.last_iterations[-2:],
                             "edges": int(2 * 1024 * 1023)}
        del sysm, bt, xs, vals
        torch.cuda.empty_cache()
    if "next" in which:
        out.update(run_next_rows(device, reps))
    return out


def batch_bytes(ns, nzs, infos, sv, nb=0, nzb=0, binfos=()):
    """Algorithmic DRAM bytes of one batched solve (value size sv: 4 for the
    FP32 inner iterations, 8 for FP64; 16-bit column offsets).

    Per inner iteration of a system (n rows, z entries): the product reads
    the matrix once, z (sv + 2), and p and y once each, 2 n sv; the alpha
    update reads d, p, r, y and writes d, r, 6 n sv; the p update reads r, p
    and writes p, 3 n sv.  Per refinement: the FP64 residual reads the FP64
    matrix, z (8 + 2), x, d, b, p and writes r, n (8 + 8 + 3 sv); the fold
    reads and writes x and d and the p update moves 3 n sv (counted with the
    iteration), n (16 + 2 sv).  The block (n_b rows, z_b entries in CSR, 32
    columns) moves its matrix once per lockstep iteration while any column
    iterates, z_b (sv + 4) + 4 n_b, and 32 x the per-row vector terms; its
    refinement events are counted as the largest column refinement count."""
    total = 0
    for n, z, inf in zip(ns, nzs, infos):
        total += inf.iterations * (z * (sv + 2) + 11 * n * sv)
        total += inf.refinements * (z * (8 + 2) + n * (16 + 3 * sv) + n * (16 + 2 * sv))
    if binfos:
        its = max(i.iterations for i in binfos)
        refs = max(i.refinements for i in binfos)
        total += its * (nzb * (sv + 4) + 4 * nb + 32 * 11 * nb * sv)
        total += refs * (nzb * (8 + 4) + 4 * nb + 32 * nb * (16 + 3 * sv + 16 + 2 * sv))
    return total


def run_c4(device: int, reps: int):
    """The batched workload: 256 k-NN Laplacians of 4,096..131,072 rows and a
    32-column block of right-hand sides for system 0, every system and column
    to ||b - A x|| / ||b|| < 1e-10 in one cooperative launch; FP32 inner
    iterations with FP64 refinement against the same kernel in FP64.  Each
    precision runs with the launch shape the library's autotuner picks for
    it."""
    import torch
    import spmv_b200 as S
    from spmv_b200 import gen
    from spmv_b200.core import Batch
    hbm, src = peaks()
    t0 = time.perf_counter()
    systems = gen.c4_systems(count=256)
    gen_s = time.perf_counter() - t0
    n0 = systems[0][0].nrows
    Bh = gen.c4_block_rhs(n0)
    comm = S.Comm(size=1, device=device)
    stream = comm.torch_stream()
    t0 = time.perf_counter()
    B = Batch(comm, [(A.rowptr, A.cols, A.vals) for A, _ in systems], block=(0, 32))
    create_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    tune = {p: B.autotune(p) for p in ("mixed", "fp64")}
    tune_s = time.perf_counter() - t0
    bb = [torch.from_numpy(b).cuda(device) for _, b in systems]
    Bd = torch.from_numpy(Bh).cuda(device)
    ns = [A.nrows for A, _ in systems]
    nzs = [A.nnz for A, _ in systems]
    nzb = systems[0][0].nnz
    st = B.stats()
    res = {}
    sols = {}
    for prec, sv in (("mixed", 4), ("fp64", 8)):
        # One untimed solve first (the first after the autotuner's shapes runs
        # about 50 ms longer), then each solve timed on its own with CUDA
        # events; the median is reported and every time listed.
        B.solve(bb, 20000, 1e-10, block_b=Bd, precision=prec)
        times = []
        for _ in range(max(reps, 3)):
            ti, (x, info, X, binfo) = _timed(
                stream, lambda: B.solve(bb, 20000, 1e-10, block_b=Bd, precision=prec), 1)
            times.append(ti)
        t = float(np.median(times))
        byts = batch_bytes(ns, nzs, info, sv, n0, nzb, binfo)
        allinfo = list(info) + list(binfo)
        res[prec] = {
            "ms_per_launch": t * 1e3, "ms_each": [round(v * 1e3, 2) for v in times],
            "launches_per_s": 1.0 / t,
            "rhs_solves_per_s": len(allinfo) / t,
            "inner_iterations_total": sum(i.iterations for i in allinfo),
            "refinements_total": sum(i.refinements for i in allinfo),
            "max_iterations": max(i.iterations for i in allinfo),
            "converged": sum(int(i.converged) for i in allinfo),
            "worst_relres": max(i.relres for i in allinfo),
            "bytes_per_launch": byts, "gbs": byts / t / 1e9,
            "frac_of_measured_hbm": byts / t / 1e9 / hbm,
            "config": tune[prec]}
        sols[prec] = ([v.clone() for v in x], X.clone())
    err = max(float(torch.linalg.norm(a - b) / torch.linalg.norm(b))
              for a, b in zip(sols["mixed"][0] + [sols["mixed"][1]],
                              sols["fp64"][0] + [sols["fp64"][1]]))
    return {"systems": len(systems), "rows": st["rows"], "nnz": st["nnz"],
            "stored_entries": st["stored"], "index_bits": st["index_bits"],
            "block": {"system": 0, "rows": n0, "rhs": 32},
            "rhs_per_launch": len(systems) + 32,
            "mixed": res["mixed"], "fp64": res["fp64"],
            "speedup_mixed_vs_fp64": res["fp64"]["ms_per_launch"] / res["mixed"]["ms_per_launch"],
            "max_rel_diff_mixed_vs_fp64_solution": err,
            "peak_source": src, "h_mean": float(np.mean([A.scalar for A, _ in systems])),
            "generation_s": gen_s, "create_s": create_s, "autotune_s": tune_s}


def run_next_rows(device: int, reps: int):
    """The rows beyond the CG path, on the c2 matrix (3D 7-point 128^3, 8
    ranks): complex128 Matrix::mult (GB/s against the measured HBM peak),
    the PETSc binary reader (file written untimed, read timed, host), and
    create_matrix on a 5-point assembly of a 512^2 node grid over 8 ranks,
    each rank also holding the next grid line's rows (host)."""
    import tempfile
    import torch
    import spmv_b200 as S
    from spmv_b200 import gen, petsc
    out = {}
    hbm, src = peaks()
    W = gen.workload(WORKLOAD)
    D = gen.distribute(W.A, W.P)
    P = W.P
    n, nnz = W.A.nrows, W.A.nnz
    g = int(sum(len(x) for x in D.ghosts))
    # complex128 mult -----------------------------------------------------
    comm = S.Comm(size=P, device=device)
    stream = comm.torch_stream()
    cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
    rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(P)])
    rng = np.random.default_rng(12)
    blocks = [(rp, ci, (va + 1j * rng.standard_normal(len(va))).astype(np.complex128))
              for rp, ci, va in D.blocks]
    Mc = S.Matrix(comm, blocks, cm, rm)
    Mc.autotune(reps=5)
    xs = [torch.complex(torch.rand(cm.vec_len(q), dtype=torch.float64, device=f"cuda:{device}"),
                        torch.rand(cm.vec_len(q), dtype=torch.float64, device=f"cuda:{device}"))
          for q in range(P)]
    ys = [torch.empty(D.local_sizes[q], dtype=torch.complex128, device=f"cuda:{device}")
          for q in range(P)]
    t, _ = _timed(stream, lambda: Mc.mult(xs, out=ys), max(reps, 20))
    kb = kernel_bytes(n, nnz, P, g, sv=16)
    out["complex128_mult_c2"] = {"us_per_launch": t * 1e6, "bytes_per_launch": kb,
                                 "gbs": kb / t / 1e9, "frac_of_measured_hbm": kb / t / 1e9 / hbm,
                                 "kernel": Mc.get_kernel()}
    del Mc, xs, ys, blocks
    torch.cuda.empty_cache()
    # Restriction: restrictmain.cpp:56-88's loop body on the c2 operator ---
    # psp = R.transpmult(q) (Matrix.cpp:168-176), then reverse_update(psp)
    # (L2GMap.cpp:152-170): the ghost entries of each rank's A^T q are added
    # into their owners.
    comm = S.Comm(size=P, device=device)
    stream = comm.torch_stream()
    cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
    rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(P)])
    Mr = S.Matrix(comm, D.blocks, cm, rm)
    dev = f"cuda:{device}"
    qs = [torch.rand(D.local_sizes[r], dtype=torch.float64, device=dev) for r in range(P)]
    ps = [torch.empty(cm.vec_len(r), dtype=torch.float64, device=dev) for r in range(P)]
    for _ in range(3):
        Mr.transpmult(qs, out=ps)
        cm.reverse_update(ps)
    nr = max(reps, 50)
    t_tm, _ = _timed(stream, lambda: Mr.transpmult(qs, out=ps), nr)
    t_ru, _ = _timed(stream, lambda: cm.reverse_update(ps), nr)
    t_both, _ = _timed(stream, lambda: (Mr.transpmult(qs, out=ps), cm.reverse_update(ps)), nr)
    # Algorithmic bytes: A^T as CSR (values, columns, row pointers), q read
    # once, A^T q written once (owned + ghost entries); reverse_update reads
    # each ghost value and its owner's entry and writes the owner's entry,
    # with one 4-byte index per contribution and per target.
    tb = nnz * 12 + (n + g + P) * 4 + n * 8 + (n + g) * 8
    rb = g * (8 + 4) + g * (8 + 8 + 4)
    out["restrict_c2"] = {
        "transpmult_us": t_tm * 1e6, "transpmult_bytes": tb,
        "transpmult_gbs": tb / t_tm / 1e9, "transpmult_frac_of_measured_hbm": tb / t_tm / 1e9 / hbm,
        "reverse_update_us": t_ru * 1e6, "reverse_update_bytes": rb,
        "reverse_update_gbs": rb / t_ru / 1e9,
        "transpmult_plus_reverse_update_us": t_both * 1e6,
        "transpmult_plus_reverse_update_gbs": (tb + rb) / t_both / 1e9,
        "frac_of_measured_hbm": (tb + rb) / t_both / 1e9 / hbm}
    del Mr, qs, ps
    torch.cuda.empty_cache()
    # PETSc reader ----------------------------------------------------------
    with tempfile.TemporaryDirectory() as d:
        fa = f"{d}/A.dat"
        petsc.write_matrix(fa, W.A.rowptr, W.A.cols, W.A.vals, W.A.ncols)
        size = os.path.getsize(fa)
        t0 = time.perf_counter()
        A = S.read_petsc_binary(S.Comm(size=P, device=device), fa)
        tr = time.perf_counter() - t0
        same = all(np.array_equal(A.mat(q)[1], D.blocks[q][1]) for q in range(P))
        out["petsc_read_c2"] = {"seconds": tr, "file_bytes": size,
                                "file_mb_per_s": size / tr / 1e6,
                                "blocks_equal_workload_distribution": bool(same)}
        del A
    # create_matrix -----------------------------------------------------------
    nx = 512
    nodes = nx * nx
    bl, nrl, rgs, cgs = gen.grid_assembly_5pt(nx, P)
    S.create_matrix(S.Comm(size=P, device=device), bl, nrl, nrl, rgs, cgs)  # warm the path
    t0 = time.perf_counter()
    Ma = S.create_matrix(S.Comm(size=P, device=device), bl, nrl, nrl, rgs, cgs)
    ta = time.perf_counter() - t0
    t0 = time.perf_counter()
    S.create_matrix(S.Comm(size=P, device=-1), bl, nrl, nrl, rgs, cgs)
    th = time.perf_counter() - t0
    out["create_matrix_512sq"] = {"seconds": ta, "host_assembly_seconds": th, "rows": nodes,
                                   "entries_in": int(sum(len(b[1]) for b in bl)),
                                   "entries_out": int(sum(Ma.nnz(q) for q in range(P)))}
    return out


# ---------------------------------------------------------------------------
# Reference arm
# ---------------------------------------------------------------------------
def run_reference(args, world, rank):
    """The reference's CPU path on this host: each step is one complete FP64
    CG solve of the workload by the oracle's restatement of spmv::cg
    (cg.cpp:11-83) on all host threads (MKL, Eigen and MPI are not available
    to build the reference itself)."""
    if rank != 0:
        return
    from spmv_b200 import gen
    import oracle
    W = gen.workload(WORKLOAD)
    D = gen.distribute(W.A, W.P)
    nthreads = oracle.max_threads()
    per_step, its = [], []
    for i in range(args.warmup + args.steps):
        dt, k = cpu_full_solve(W, D, nthreads)
        if i >= args.warmup:
            per_step.append(dt)
            its.append(k)
    t = float(np.mean(per_step))
    value = 1.0 / t
    sample = ("oracle spmv::cg restatement (reference-restatement CPU, not MKL), "
              "%d threads on %s: every step one complete solve (%d iterations)"
              % (nthreads, cpu_model(), its[0]))
    line = {"impl": "reference", "metric": "CG solves/s", "value": value,
            "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": config_dict(W, D, W.P),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": nthreads,
                             "kind": "port", "sample": sample, "cpu_model": cpu_model()},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(args, info):
    import torch
    import spmv_b200 as S
    world, rank, device = info.world, info.rank, info.local
    torch.cuda.set_device(device)
    W, D, comm, cm, rm, M = setup(device)
    P = W.P
    stream = torch.cuda.ExternalStream(comm.stream, device=f"cuda:{device}")
    n, nnz = W.A.nrows, W.A.nnz
    g = int(sum(len(x) for x in D.ghosts))

    # Device-resident inputs.
    bd = [torch.from_numpy(W.b[D.ranges[q]:D.ranges[q + 1]].copy()).cuda(device)
          for q in range(P)]
    xd = [torch.zeros(cm.vec_len(q), dtype=torch.float64, device=f"cuda:{device}")
          for q in range(P)]

    # --- value: K device-resident solves ---------------------------------
    k_its = None
    for _ in range(args.warmup):
        _, k_its = S.cg(comm, M, bd, 10000, W.rtol, x=xd)
    clocks = ClockSampler(device)
    barrier(info)
    clocks.start()
    t_ev0 = torch.cuda.Event(enable_timing=True)
    t_ev1 = torch.cuda.Event(enable_timing=True)
    t_ev0.record(stream)
    its = []
    for _ in range(args.steps):
        _, k = S.cg(comm, M, bd, 10000, W.rtol, x=xd)
        its.append(k)
    t_ev1.record(stream)
    torch.cuda.synchronize(device)
    clk = clocks.stop()
    barrier(info)
    t_local = t_ev0.elapsed_time(t_ev1) / 1e3
    t_max = max_over_ranks(t_local, info)
    value = world * args.steps / t_max
    k_mean = float(np.mean(its))

    # --- e2e: the same solve with pinned host buffers through the C ABI ----
    bh = [torch.from_numpy(W.b[D.ranges[q]:D.ranges[q + 1]].copy()).pin_memory().numpy()
          for q in range(P)]
    xh = [torch.zeros(cm.vec_len(q), dtype=torch.float64).pin_memory().numpy()
          for q in range(P)]
    S.cg(comm, M, bh, 10000, W.rtol, x=xh)
    barrier(info)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        S.cg(comm, M, bh, 10000, W.rtol, x=xh)
    e1.record(stream)
    torch.cuda.synchronize(device)
    barrier(info)
    te = max_over_ranks(e0.elapsed_time(e1) / 1e3, info)
    e2e = world * args.steps / te
    h2d = int(sum(v.nbytes for v in bh))
    d2h = int(sum(D.local_sizes[q] * 8 for q in range(P)))

    # --- roofline of the product kernel (matvec loop: update + mult) -------
    xs = [torch.rand(cm.vec_len(q), dtype=torch.float64, device=f"cuda:{device}")
          for q in range(P)]
    ys = [torch.empty(D.local_sizes[q], dtype=torch.float64, device=f"cuda:{device}")
          for q in range(P)]
    reps = args.spmv_reps
    for _ in range(5):
        cm.update(xs)
        M.mult(xs, out=ys)
    barrier(info)
    # The reps are queued behind a spin kernel, so the host has issued all of
    # them before the first runs and the events bracket GPU work only (a
    # Python call costs about as much host time as one launch takes).
    a0, a1, a2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    torch.cuda.synchronize(device)
    with torch.cuda.stream(stream):
        torch.cuda._sleep(100_000_000)  # ~50 ms at B200 clocks
        a0.record(stream)
        for _ in range(reps):
            M.mult(xs, out=ys)
        a1.record(stream)
        for _ in range(reps):
            cm.update(xs)
            M.mult(xs, out=ys)
        a2.record(stream)
    torch.cuda.synchronize(device)
    t_mult = a0.elapsed_time(a1) / 1e3 / reps
    t_pair = a1.elapsed_time(a2) / 1e3 / reps
    hbm, src = peaks()
    kb = kernel_bytes(n, nnz, P, g)
    achieved = kb / t_mult / 1e9
    sb = spmv_bytes(n, nnz, P, g)
    kname, kwidth, kblock = M.get_kernel()
    kernel_fn = {"sell": "spmv_sell_kernel", "vector": "spmv_vector_kernel",
                 "staged": "spmv_staged_kernel",
                 "merge": "merge_kernel"}.get(kname, kname)
    traffic = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        try:
            traffic = json.loads(tp.read_text()).get(f"{kernel_fn}_c2")
        except Exception:
            traffic = None

    # CG iteration bytes (fused-halo layout: no ghost gather, 9 n vector terms),
    # counted for 32-bit CSR; the product may store its columns as 16-bit
    # offsets, which moves 2 bytes less per nonzero than counted.
    b_iter = kernel_bytes(n, nnz, 1, 0) + 9 * n * 8
    cg_kind, cg_w, cg_bits, cg_us = M.solver_product("cg")
    cg_form = M.cg_form()
    ms_per_iter = t_local / args.steps / k_mean * 1e3

    # Roofline of the kernel that runs the timed steps.  A fused solve is one
    # cooperative launch per step, so its duration is the step time;
    # algorithmic bytes = B_iter x iterations.  The vectors stay in L2 (and
    # r in shared memory), so DRAM carries little more than the matrix:
    # "dram_frac" is the matrix stream's bytes over the same time.
    mult_roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                 "frac": achieved / hbm, "peak_source": src, "traffic": traffic,
                 "traffic_source": "profiles/traffic.json (committed ncu capture)",
                 "kernel": f"{kernel_fn} width={kwidth} block={kblock} "
                           "(Matrix::mult, 8 ranks, one launch)",
                 "bytes_per_launch": kb, "us_per_launch": t_mult * 1e6}
    cg_roof = None
    if cg_form[0] == "fused":
        t_launch = t_local / args.steps
        cg_bytes = b_iter * k_mean
        cg_ach = cg_bytes / t_launch / 1e9
        matrix_bytes = nnz * (8 + cg_bits // 8) * k_mean
        cg_traffic = None
        if tp.exists():
            try:
                merged = bool(cg_form[2] and cg_form[2].endswith(":m"))
                cg_traffic = json.loads(tp.read_text()).get(
                    "cg_fused_merged_c2" if merged else "cg_fused_c2")
            except Exception:
                cg_traffic = None
        # achieved / frac count the compulsory DRAM bytes: the matrix stream
        # at its stored index width, once per iteration (the CG vectors, 84 MB,
        # stay in L2 and r in shared memory); the B_iter figure, which counts
        # vector traffic that never reaches DRAM, is kept as algorithmic_gbs.
        mat_ach = matrix_bytes / t_launch / 1e9
        cg_roof = {"bound": "hbm", "achieved": mat_ach, "peak": hbm, "unit": "GB/s",
                   "frac": mat_ach / hbm, "peak_source": src, "traffic": cg_traffic,
                   "traffic_source": "profiles/traffic.json: dram__bytes_read.sum + "
                                     "dram__bytes_write.sum of one launch, committed ncu "
                                     "capture (not measured in this run)",
                   "kernel": f"cg_fused ({cg_form[1]} CTAs/SM, r in {cg_form[2].split(':')[0]}, "
                             f"staged width {cg_w}, {cg_bits}-bit indices, "
                             f"{2 if cg_form[2].endswith(':m') else 3} grid syncs per "
                             "iteration; one launch per solve)",
                   "bytes_per_launch": matrix_bytes, "us_per_launch": t_launch * 1e6,
                   "bytes_model": "nnz x (8 + index bytes) x iterations",
                   "algorithmic_gbs": cg_ach, "algorithmic_bytes_per_launch": cg_bytes}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        import oracle
        nth = oracle.max_threads()
        dt, kf = cpu_full_solve(W, D, nth)
        spi1, k1 = cpu_sample(W, D, args.cpu_budget, 1)
        cpu = {"value": 1.0 / dt, "unit": "solves/s", "cores": nth, "kind": "port",
               "cpu_model": cpu_model(),
               "sample": "oracle spmv::cg restatement (reference-restatement CPU, not MKL) "
                         "on %d host threads: one complete solve (%d iterations, %.1f s)"
                         % (nth, kf, dt),
               "single_thread": {"value": 1.0 / (spi1 * kf), "unit": "solves/s", "cores": 1,
                                 "sample": "%d CG iterations at 1 thread (%.1f s; the "
                                           "reference CI runs OMP_NUM_THREADS=1), scaled to "
                                           "the %d iterations of a full solve"
                                           % (k1, spi1 * k1, kf)}}

    extras = None
    if world == 1 and not args.no_extras:
        extras = run_extras(device, args.extra_reps, args.c4_count,
                            tuple(args.extras.split(",")))

    if rank == 0:
        line = {
            "metric": "CG solves/s", "value": value, "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": config_dict(W, D, P),
            "roofline": cg_roof if cg_roof is not None else mult_roof,
            "mult_roofline": mult_roof,
            "spmv": {"update_plus_mult_gbs": sb / t_pair / 1e9,
                     "update_plus_mult_us": t_pair * 1e6, "bytes": sb,
                     "frac_of_measured_hbm": sb / t_pair / 1e9 / hbm,
                     "frac_of_8TBs": sb / t_pair / 1e9 / 8000.0},
            "cg": {"iterations": k_mean, "ms_per_iter": ms_per_iter,
                   "gbs": b_iter / (ms_per_iter / 1e3) / 1e9,
                   "bytes_per_iter": b_iter,
                   "product": {"kernel": cg_kind, "width": cg_w, "index_bits": cg_bits,
                               "plain_us": cg_us},
                   "form": {"kind": cg_form[0], "ctas_per_sm": cg_form[1],
                            "residual_in": cg_form[2] and cg_form[2].split(":")[0],
                            "merged_update": bool(cg_form[2] and cg_form[2].endswith(":m"))}},
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            # A graph solve launches an init kernel and three per iteration;
            # a fused solve is one cooperative launch.
            "gpu_launches": int(args.steps * (1 if cg_form[0] == "fused" else 1 + 3 * k_mean)),
            "clocks": clk,
        }
        if cpu:
            line["cpu_baseline"] = cpu
        if extras:
            line["extras"] = extras
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Per-configuration table (--table): the CPU restatement beside the GPU path
# ---------------------------------------------------------------------------
def run_table(args):
    """For c1, c2, c3 and c5 at full size, one JSON line each and a markdown
    table: SpMV GB/s (B_spmv over one L2GMap::update + Matrix::mult) and CG
    solves/s, on the GPU (autotuned product; L2 flushed between SpMV reps
    for the configurations that fit in L2) and for the oracle's restatement
    on all host threads (SpMV: best of repeated update + mult; CG: a bounded
    run of iterations scaled to the GPU's iteration count)."""
    import torch
    import spmv_b200 as S
    import oracle
    from spmv_b200 import gen
    nth = oracle.max_threads()
    dev = torch.device("cuda:0")
    flush = torch.ones(256 << 20, dtype=torch.uint8, device=dev)  # > 126 MB L2
    rows = []
    for name in ("c1", "c2", "c3", "c5"):
        W = gen.workload(name)
        D = gen.distribute(W.A, W.P)
        P, n, nnz = W.P, W.A.nrows, W.A.nnz
        g = int(sum(len(x) for x in D.ghosts))
        B = spmv_bytes(n, nnz, P, g)
        comm = S.Comm(size=P, device=0)
        cm = S.L2GMap(comm, D.local_sizes, D.ghosts)
        rm = S.L2GMap(comm, D.local_sizes, [[] for _ in range(P)])
        M = S.Matrix(comm, D.blocks, cm, rm)
        M.autotune(reps=10)
        stream = torch.cuda.ExternalStream(comm.stream, device=dev)
        resident = B < 100e6
        xs = [torch.rand(cm.vec_len(q), dtype=torch.float64, device=dev) for q in range(P)]
        ys = [torch.empty(D.local_sizes[q], dtype=torch.float64, device=dev) for q in range(P)]
        for _ in range(3):
            cm.update(xs)
            M.mult(xs, out=ys)
        # Reps queued behind a spin kernel, so the host has issued all of
        # them before the first runs; each rep's update + mult is bracketed
        # by its own events (GPU time alone).  For the L2-resident
        # configurations each rep follows a read of 256 MB, which leaves the
        # L2 holding other, clean lines.
        R = 50
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(R)]
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            torch.cuda._sleep(200_000_000)  # ~0.1 s at B200 clocks
            for i in range(R):
                if resident:
                    flush.sum(dtype=torch.int64)
                ev[i][0].record(stream)
                cm.update(xs)
                M.mult(xs, out=ys)
                ev[i][1].record(stream)
        torch.cuda.synchronize()
        times = [a.elapsed_time(b) / 1e3 for a, b in ev]
        gpu_spmv = B / statistics.median(times) / 1e9
        # GPU CG: device-resident b and x, the configuration's tolerance.
        bd = [torch.from_numpy(W.b[D.ranges[q]:D.ranges[q + 1]].copy()).to(dev)
              for q in range(P)]
        xd = [torch.zeros(cm.vec_len(q), dtype=torch.float64, device=dev) for q in range(P)]
        _, k = S.cg(comm, M, bd, 20000, W.rtol, x=xd)
        reps = 3 if n < 3_000_000 else 1
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            S.cg(comm, M, bd, 20000, W.rtol, x=xd)
        e1.record(stream)
        torch.cuda.synchronize()
        gpu_cg = reps / (e0.elapsed_time(e1) / 1e3)
        # CPU restatement: update + mult over all ranks, then a CG sample.
        om = oracle.Map(D.local_sizes, D.ghosts)
        xh = [np.random.default_rng(q).uniform(-1, 1, cm.vec_len(q)) for q in range(P)]
        cpu_t = []
        t_end = time.perf_counter() + min(5.0, args.cpu_budget)
        while time.perf_counter() < t_end or len(cpu_t) < 3:
            t0 = time.perf_counter()
            om.update(xh)
            for q in range(P):
                rp, ci, va = D.blocks[q]
                oracle.csr_mult(rp, ci, va, xh[q], nthreads=nth)
            cpu_t.append(time.perf_counter() - t0)
        cpu_spmv = B / min(cpu_t) / 1e9
        spi, kk = cpu_sample(W, D, args.cpu_budget, nth)
        cpu_cg = 1.0 / (spi * k)
        row = {"config": name, "n": n, "nnz": nnz, "ranks": P, "cg_iterations": int(k),
               "cg_form": list(M.cg_form()), "mult_kernel": list(M.get_kernel()),
               "cpu_spmv_gbs": cpu_spmv, "cpu_cg_solves_per_s": cpu_cg, "cpu_threads": nth,
               "cpu_cg_sample_iterations": kk, "gpu_spmv_gbs": gpu_spmv,
               "gpu_cg_solves_per_s": gpu_cg, "l2": "flushed" if resident else "exceeded"}
        rows.append(row)
        print(json.dumps(row), flush=True)
        M.close()
        cm.close()
        rm.close()
        comm.close()
    print("| cfg | CPU SpMV GB/s | CPU CG solves/s | cores | GPU SpMV GB/s | GPU CG solves/s |")
    print("|---|---|---|---|---|---|")
    for r in rows:
        print("| %s | %.1f | %.4g | %d | %.0f | %.4g |" % (
            r["config"], r["cpu_spmv_gbs"], r["cpu_cg_solves_per_s"], r["cpu_threads"],
            r["gpu_spmv_gbs"], r["gpu_cg_solves_per_s"]))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--spmv-reps", type=int, default=200)
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--ref-budget", type=float, default=1.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the c3/c4/c5 mixed, batched and adjoint measurements")
    ap.add_argument("--extra-reps", type=int, default=2)
    ap.add_argument("--c4-count", type=int, default=256)
    ap.add_argument("--extras", default="c3,c2,c4,c5,next",
                    help="comma-separated parts of the extras: c3, c2, c4, c5, next")
    ap.add_argument("--table", action="store_true",
                    help="per-configuration CPU/GPU table (c1, c2, c3, c5) instead of the "
                         "benchmark line")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    info = dist_init()
    try:
        if args.table:
            if info.rank == 0:
                run_table(args)
        elif args.impl == "reference":
            run_reference(args, info.world, info.rank)
        else:
            run_ours(args, info)
    finally:
        from spmv_b200 import ranks
        ranks.finalize(info)


if __name__ == "__main__":
    main()
