"""The C ABI library loads on a machine without a GPU and exports every entry
point include/spmv_b200.h declares; host-only calls work and device calls fail
with a status instead of crashing."""
import ctypes as C

import numpy as np
import pytest

from spmv_b200 import _lib
import spmv_b200 as S


def test_exports_every_declared_symbol():
    L = _lib.lib()
    names = _lib.declared_symbols()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert missing == []


def test_python_binding_covers_header():
    names = set(_lib.declared_symbols())
    bound = set(_lib._SIGS) | {"spmv_last_error"}
    assert names <= bound, sorted(names - bound)


def test_version_and_last_error():
    ma, mi = C.c_int(), C.c_int()
    _lib.call("spmv_get_version", C.byref(ma), C.byref(mi))
    assert (ma.value, mi.value) == (0, 1)
    st = _lib.lib().spmv_comm_create(-1, None, 0, C.byref(C.c_void_p()))
    assert st == _lib.ERROR_INVALID_ARGUMENT
    assert "size" in _lib.lib().spmv_last_error().decode()


def test_host_only_comm_refuses_device_work():
    comm = S.Comm(size=2, device=-1)
    m = S.L2GMap(comm, [3, 3], [[3], [2]])
    with pytest.raises(S.SpmvError) as e:
        m.update([np.zeros(4), np.zeros(4)])
    assert e.value.status == _lib.ERROR_NO_DEVICE
    with pytest.raises(S.SpmvError):
        comm.synchronize()


def test_null_handles_are_errors():
    L = _lib.lib()
    out = C.c_int32()
    assert L.spmv_l2gmap_local_size(None, 0, C.byref(out)) == _lib.ERROR_INVALID_ARGUMENT
    assert L.spmv_matrix_mult(None, 0, None, None) == _lib.ERROR_INVALID_ARGUMENT
    assert L.spmv_comm_destroy(None) == _lib.SUCCESS


def test_matrix_validation_messages():
    comm = S.Comm(size=1, device=-1)
    cm = S.L2GMap(comm, [3], [[]])
    rp = np.array([0, 1, 2, 3], np.int32)
    with pytest.raises(S.SpmvError, match="column index out of range"):
        S.Matrix(comm, [(rp, np.array([0, 1, 3], np.int32), np.ones(3))], cm, cm)
    with pytest.raises(S.SpmvError, match="non-decreasing"):
        S.Matrix(comm, [(np.array([0, 2, 1, 3], np.int32), np.zeros(3, np.int32),
                         np.ones(3))], cm, cm)
    with pytest.raises(S.SpmvError, match="ncols"):
        S.Matrix(comm, [(rp, np.zeros(3, np.int32), np.ones(3))], cm, cm, ncols=[4])
    A = S.Matrix(comm, [(rp, np.array([0, 1, 2], np.int32), np.ones(3))], cm, cm)
    rpa, cia, vaa = A.mat(0)
    assert np.array_equal(rpa, rp) and np.array_equal(cia, [0, 1, 2])
    assert np.array_equal(vaa, np.ones(3))
    assert A.get_kernel() == ("vector", 1, 256) or A.get_kernel()[0] == "vector"


def test_destroy_order_does_not_matter():
    # The communicator and maps are reference counted by what uses them, as
    # the reference's Matrix holds its maps by shared_ptr.
    L = _lib.lib()
    comm = C.c_void_p()
    _lib.call("spmv_comm_create", -1, None, 1, C.byref(comm))
    ls = (C.c_int64 * 1)(3)
    g = (C.POINTER(C.c_int64) * 1)()
    ng = (C.c_int64 * 1)(0)
    cm = C.c_void_p()
    _lib.call("spmv_l2gmap_create", comm, ls, g, ng, C.byref(cm))
    rp = np.array([0, 1, 2, 3], np.int32)
    ci = np.array([0, 1, 2], np.int32)
    va = np.ones(3)
    A = C.c_void_p()
    _lib.call("spmv_matrix_create_csr", comm, _lib.FLOAT64, cm, cm, (C.c_int32 * 1)(3),
              (C.c_int32 * 1)(3), _lib.ptr_array([rp.ctypes.data]),
              _lib.ptr_array([ci.ctypes.data]), _lib.ptr_array([va.ctypes.data]),
              C.byref(A))
    assert L.spmv_comm_destroy(comm) == 0
    assert L.spmv_l2gmap_destroy(cm) == 0
    n = C.c_int64()
    _lib.call("spmv_matrix_nnz", A, 0, C.byref(n))  # still usable
    assert n.value == 3
    m = C.c_void_p()
    _lib.call("spmv_matrix_col_map", A, C.byref(m))
    gs = C.c_int64()
    _lib.call("spmv_l2gmap_global_size", m, C.byref(gs))
    assert gs.value == 3
    assert L.spmv_matrix_destroy(A) == 0
