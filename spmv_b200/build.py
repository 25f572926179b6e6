"""Build recipe for the native libraries of spmv_b200 (in-tree).

* ``spmv_b200/libspmv_b200.so`` - the CUDA library behind include/spmv_b200.h,
  compiled for sm_100a only.
* ``spmv_b200/libspmv_gen.so`` - host generators of the synthetic workloads.

Objects go to ``spmv_b200/_build``.  A library is rebuilt when any of its
sources or headers is newer than it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = PKG / "_build"

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: vector updates round their products and sums separately, as the
# reference's Eigen expressions do on x86-64 without FMA.
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-fmad=false",
                     "-Xcompiler", "-fPIC,-O3", "-I" + str(INCLUDE),
                     "-I" + str(CSRC)]
CXX = "g++"  # the system compiler (has OpenMP)

LIB = PKG / "libspmv_b200.so"
GEN = PKG / "libspmv_gen.so"

CUDA_SOURCES = ["api.cpp", "l2gmap.cpp", "spmv.cu", "merge.cu", "halo.cu", "cg.cu", "ir.cu", "adjoint.cu", "sell.cu", "batch.cu", "batch_plan.cpp", "batch_f32.cu", "batch_f64.cu", "tune.cpp", "block.cu", "petsc.cpp", "assemble.cpp", "assemble_dev.cu"]
HEADERS = ["internal.h", "kernels.cuh", "spmv_kernel.cuh", "sell_staged.cuh", "batch.h",
           "batch_kernel.cuh"]


def _newer(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: " + " ".join(map(str, cmd)) + "\n" +
                           r.stdout + r.stderr)
    return r


def build_lib(force: bool = False, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    headers = [CSRC / h for h in HEADERS] + [INCLUDE / "spmv_b200.h"]
    objs, jobs = [], []
    for src in CUDA_SOURCES:
        s = CSRC / src
        o = BUILD / (src + ".o")
        objs.append(o)
        if force or _newer(o, [s] + headers):
            cmd = [NVCC] + NVCC_FLAGS + ["-c", str(s), "-o", str(o)]
            if src.endswith(".cu") and verbose:
                cmd += ["-Xptxas", "-v"]
            jobs.append(cmd)
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for r in ex.map(_run, jobs):
            if verbose:
                print(r.stdout + r.stderr)
    if force or jobs or _newer(LIB, objs):
        tmp = LIB.with_suffix(".so.tmp")
        _run([NVCC] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs])
        os.replace(tmp, LIB)  # readers never see a half-written library
    return LIB


def build_gen(force: bool = False) -> Path:
    src = CSRC / "gen.cpp"
    if force or _newer(GEN, [src, CSRC / "spmv_gen.h"]):
        tmp = GEN.with_suffix(".so.tmp")
        _run([CXX, "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared",
              "-I" + str(CSRC), str(src), "-o", str(tmp)])
        os.replace(tmp, GEN)
    return GEN


def build(force: bool = False, verbose: bool = False) -> None:
    build_gen(force)
    build_lib(force, verbose)


if __name__ == "__main__":
    import sys
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print("built", LIB, GEN)
