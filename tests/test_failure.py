"""Host-side fault injection: invalid inputs, invalid plans and calls out of order come back as
error statuses with a message (the reference exits the process after cudaDeviceReset on CUDA
errors, include/cytnx_error.hpp:519-536; here nothing resets a device).  No GPU is needed: every
case is rejected before any device work."""
import ctypes

import numpy as np
import pytest
import torch

from cytnx_b200 import _lib
from cytnx_b200 import workloads as W


def _status(fn, *args):
    st = fn(*args)
    return st, _lib.lib().ctn_last_error().decode()


def test_permute_rejects_bad_mapper_and_dtype():
    lib = _lib.lib()
    shape = np.array([2, 3, 4], dtype=np.uint64)
    dup = np.array([0, 0, 2], dtype=np.uint64)
    st, msg = _status(lib.ctn_permute, None, None, 3, 3, shape.ctypes.data_as(_lib.P_u64),
                      dup.ctypes.data_as(_lib.P_u64), None)
    assert st != 0 and "invalid mapper" in msg
    oob = np.array([0, 1, 7], dtype=np.uint64)
    st, msg = _status(lib.ctn_permute, None, None, 3, 3, shape.ctypes.data_as(_lib.P_u64),
                      oob.ctypes.data_as(_lib.P_u64), None)
    assert st != 0 and "invalid mapper" in msg
    ok = np.array([2, 1, 0], dtype=np.uint64)
    st, msg = _status(lib.ctn_permute, None, None, 99, 3, shape.ctypes.data_as(_lib.P_u64),
                      ok.ctypes.data_as(_lib.P_u64), None)
    assert st != 0 and "unknown dtype" in msg
    st, msg = _status(lib.ctn_permute, None, None, 3, 40, shape.ctypes.data_as(_lib.P_u64),
                      ok.ctypes.data_as(_lib.P_u64), None)
    assert st != 0 and "rank" in msg


def test_heff_plan_calls_out_of_order_and_bad_tiles():
    """A planned H_eff (host planning only) refuses a matvec before its environments are
    bound, unknown precisions and unsupported tile widths."""
    from cytnx_b200.heff import plan_two_site

    psi, L, M1, M2, R = W.build_two_site(W.xxz_spec(16), W.xxz_mpo_values(1.0, 1.0), seed=0, device=-1)
    h = plan_two_site(L, M1, M2, R, psi, [])[0]
    lib = _lib.lib()
    try:
        st, msg = _status(lib.ctn_heff2_matvec, h, None, None, _lib.PREC_F64, None)
        assert st != 0 and "not bound" in msg
        st, msg = _status(lib.ctn_heff2_matvec, h, None, None, _lib.PREC_BF16X3, None)
        assert st != 0 and "not bound" in msg
        st, msg = _status(lib.ctn_heff2_matvec, h, None, None, 7, None)
        assert st != 0
        st, msg = _status(lib.ctn_heff2_set_tiles, h, _lib.PREC_BF16X3, 100, 128)
        assert st != 0 and "tile" in msg
        st, msg = _status(lib.ctn_heff2_set_tiles, h, _lib.PREC_F64, 128, 128)
        assert st != 0 and "split precision only" in msg
        st, msg = _status(lib.ctn_heff2_lanczos_refined, h, _lib.PREC_BF16X3, None, 8, 2, 1e-12, None, None, None,
                          ctypes.byref(ctypes.c_double()), ctypes.byref(ctypes.c_double()),
                          ctypes.byref(ctypes.c_int()), None, None)
        assert st != 0 and "must be bound" in msg
    finally:
        lib.ctn_heff2_plan_destroy(h)


def test_contract_plan_rejects_inconsistent_structures():
    """Invalid contraction plans: output rank that does not match the free legs, no common leg."""
    lib = _lib.lib()
    itoi = np.zeros((1, 2), dtype=np.int64)
    shapes = np.array([[2, 3]], dtype=np.int64)
    offs = np.zeros(1, dtype=np.int64)
    a = _lib.BlockDesc(2, 1, itoi.ctypes.data, shapes.ctypes.data, offs.ctypes.data, None)
    out_itoi = np.zeros((1, 3), dtype=np.int64)
    out_shapes = np.array([[2, 2, 2]], dtype=np.int64)
    o = _lib.BlockDesc(3, 1, out_itoi.ctypes.data, out_shapes.ctypes.data, offs.ctypes.data, None)
    c1 = np.array([1], dtype=np.int64)
    c2 = np.array([0], dtype=np.int64)
    plan = ctypes.c_void_p()
    st, msg = _status(lib.ctn_contract_plan_create, ctypes.byref(a), ctypes.byref(a), 1,
                      c1.ctypes.data_as(_lib.P_i64), c2.ctypes.data_as(_lib.P_i64), ctypes.byref(o), ctypes.byref(plan))
    assert st != 0 and "rank" in msg
    st, msg = _status(lib.ctn_contract_plan_create, ctypes.byref(a), ctypes.byref(a), 0,
                      c1.ctypes.data_as(_lib.P_i64), c2.ctypes.data_as(_lib.P_i64), ctypes.byref(o), ctypes.byref(plan))
    assert st != 0 and "ncomm" in msg


def test_contract_rejects_bra_with_bra():
    """Contract of two BRA legs (the reference's 'BRA can only be contracted with KET')."""
    import cytnx_b200 as c
    from cytnx_b200._lib import CytnxError

    b = c.Bond(c.BD_BRA, [[0], [1]], [2, 3])
    k = c.Bond(c.BD_KET, [[0], [1]], [2, 3])
    A = c.UniTensor([b, k], labels=["x", "y"], device=-1)
    B = c.UniTensor([b, k], labels=["x", "z"], device=-1)
    with pytest.raises(CytnxError):
        c.Contract(A, B)
