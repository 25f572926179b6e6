"""Generates tests/golden/golden.json: pseudo-known answers computed by the
oracle (the CPU restatement of the reference) and cross-checked against an
independent scipy computation before they are written.

The reference publishes no outputs and cannot be built here, so these values
pin the oracle (and through it the GPU path) to itself over time, and the
scipy cross-check ties them to an independent implementation.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from spmv_b200 import gen  # noqa: E402


def matvec_demo_scipy(N=500000, n_apply=1000):
    A = gen.create_a(N).scipy()
    z = np.arange(N) / N
    x = np.exp(-10 * (5 * (z - 0.5)) ** 2)
    for _ in range(n_apply):
        x = A @ x
    return float(x @ x)


def cg_case(name, P, scale=0):
    W = gen.workload(name, scale)
    D = gen.distribute(W.A, P)
    om = oracle.Map(D.local_sizes, D.ghosts)
    b = [W.b[D.ranges[q]:D.ranges[q + 1]].copy() for q in range(P)]
    xs, k, rn = oracle.cg(om, D.blocks, b, 10000, W.rtol)
    x = np.concatenate([xs[q][:D.local_sizes[q]] for q in range(P)])
    S = W.A.scipy()
    true_rel = float(np.linalg.norm(W.b - S @ x) / np.linalg.norm(W.b))
    assert true_rel < 10 * W.rtol, (name, true_rel)
    # Independent check: scipy CG from the same start reaches the same
    # tolerance in a similar number of iterations.
    import scipy.sparse.linalg as spla
    its = [0]
    xs_sp, info = spla.cg(S, W.b, rtol=W.rtol, atol=0.0, maxiter=10000,
                          callback=lambda _: its.__setitem__(0, its[0] + 1))
    assert info == 0 and abs(its[0] - k) <= 2, (name, its[0], k)
    assert np.linalg.norm(xs_sp - x) / np.linalg.norm(x) < 1e-5
    return {"P": P, "scale": scale, "rtol": W.rtol, "iterations": int(k),
            "xnorm2": float(x @ x), "rnorm_recursive": float(rn),
            "true_relres": true_rel, "scipy_iterations": int(its[0])}


def main():
    out = {"_doc": "pseudo-KATs from the oracle (CPU restatement of "
                   "chrisrichardson/spmv); see make_golden.py"}
    demo = {}
    ref = matvec_demo_scipy()
    for P in (1, 2):
        v = oracle.matvec_demo(P, 500000, 1000)
        assert abs(v - ref) <= 1e-12 * abs(ref), (P, v, ref)
        demo[str(P)] = v
    demo["scipy"] = ref
    out["matvec_demo_N500000_apply1000"] = demo
    out["cg"] = {
        "c1": cg_case("c1", 1),
        "c2": cg_case("c2", 8),
        "c2_scale24_P8": cg_case("c2", 8, 24),
        "c1_scale64_P3": cg_case("c1", 3, 64),
    }
    path = Path(__file__).with_name("golden.json")
    path.write_text(json.dumps(out, indent=1, sort_keys=True) + "\n")
    print(json.dumps(out, indent=1, sort_keys=True))


if __name__ == "__main__":
    main()
