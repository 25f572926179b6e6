"""The C++ mirror of the reference API (include/spmv/spmv.hpp) compiles against
the C ABI and behaves like the reference: host-only checks here, the device
path under the gpu marker."""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def wrapper_exe(tmp_path_factory):
    exe = tmp_path_factory.mktemp("cpp") / "test_wrapper"
    lib = ROOT / "spmv_b200"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + str(ROOT / "include"),
                    str(ROOT / "tests" / "cpp" / "test_wrapper.cpp"), "-L" + str(lib),
                    "-lspmv_b200", "-Wl,-rpath," + str(lib), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    return exe


def test_cpp_wrapper_host(wrapper_exe, tmp_path):
    import numpy as np
    from spmv_b200 import petsc
    rp, ci, va = [0], [], []
    for i in range(5):
        for j in (i + 1, i, i - 1):  # descending columns in the file
            if 0 <= j < 5:
                ci.append(j)
                va.append(10.0 * i + j)
        rp.append(len(ci))
    fa, fb = tmp_path / "A.dat", tmp_path / "b.dat"
    petsc.write_matrix(fa, rp, ci, va, 5)
    petsc.write_vector(fb, np.arange(5.0))
    r = subprocess.run([str(wrapper_exe), "host", str(fa), str(fb)], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK 0 failures" in r.stdout


@pytest.mark.gpu
def test_cpp_wrapper_gpu(wrapper_exe, cuda_device):
    r = subprocess.run([str(wrapper_exe), "gpu"], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "OK 0 failures" in r.stdout
