"""ctypes binding of ``libcytnx_b200.so`` (the C ABI declared in include/cytnx_b200.h).

The library is built in-tree (``python -m cytnx_b200.build``).  There is no
fallback: if the library is missing or a call fails, a ``CytnxError`` is raised.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcytnx_b200.so")

c_i32 = ctypes.c_int32
c_i64 = ctypes.c_int64
c_int = ctypes.c_int
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
c_size = ctypes.c_size_t
P_i64 = ctypes.POINTER(ctypes.c_int64)
P_u64 = ctypes.POINTER(ctypes.c_uint64)
P_i32 = ctypes.POINTER(ctypes.c_int32)
P_dbl = ctypes.POINTER(ctypes.c_double)

CTN_FLOAT64 = 3
PREC_F64, PREC_3XTF32, PREC_BF16X3 = 0, 1, 2
PRECISIONS = {"fp64": PREC_F64, "f64": PREC_F64, "3xtf32": PREC_3XTF32, "bf16x3": PREC_BF16X3}


class CytnxError(RuntimeError):
    """Error raised by the cytnx_b200 library (the analogue of cytnx::error)."""


class BlockDesc(ctypes.Structure):
    _fields_ = [("rank", c_i32), ("nblocks", c_i64), ("itoi", c_vp), ("shapes", c_vp),
                ("offs", c_vp), ("perm", c_vp)]


class Heff2Desc(ctypes.Structure):
    _fields_ = [("psi", ctypes.POINTER(BlockDesc)), ("L", ctypes.POINTER(BlockDesc)),
                ("R", ctypes.POINTER(BlockDesc)), ("M1", ctypes.POINTER(BlockDesc)),
                ("M2", ctypes.POINTER(BlockDesc)), ("out", ctypes.POINTER(BlockDesc)),
                ("M1_host", c_vp), ("M2_host", c_vp)]


class GemmTask(ctypes.Structure):
    _fields_ = [("c_off", c_i64), ("m", c_i32), ("n", c_i32), ("ldc", c_i32),
                ("pair_begin", c_i32), ("pair_count", c_i32), ("pad_", c_i32)]


class GemmPair(ctypes.Structure):
    _fields_ = [("a_off", c_i64), ("b_off", c_i64), ("k", c_i32), ("lda", c_i32),
                ("ldb", c_i32), ("flags", c_i32)]


MATVEC_FN = ctypes.CFUNCTYPE(c_int, c_vp, c_vp, c_vp, c_vp)

_SIGS = {
    "ctn_last_error": (ctypes.c_char_p, []),
    "ctn_version": (c_int, []),
    "ctn_dtype_size": (c_size, [c_int]),
    "ctn_permute": (c_int, [c_vp, c_vp, c_int, c_int, P_u64, P_u64, c_vp]),
    "ctn_permute_blocks": (c_int, [c_vp, c_vp, c_int, c_int, c_i64, P_u64, P_i64, P_i64, P_u64, c_vp]),
    "ctn_blocks_enumerate": (c_int, [c_int, c_int, P_i32, P_i64, P_i32, P_i64, ctypes.POINTER(c_vp),
                                     P_i64, c_i64, P_i64]),
    "ctn_contract_plan_create": (c_int, [ctypes.POINTER(BlockDesc), ctypes.POINTER(BlockDesc), c_int,
                                         P_i64, P_i64, ctypes.POINTER(BlockDesc), ctypes.POINTER(c_vp)]),
    "ctn_contract_plan_scratch_bytes": (c_size, [c_vp]),
    "ctn_contract_plan_flops": (c_dbl, [c_vp]),
    "ctn_contract_execute": (c_int, [c_vp, c_int, c_vp, c_vp, c_vp, c_vp, c_vp]),
    "ctn_contract_plan_destroy": (None, [c_vp]),
    "ctn_gemm_grouped_plan_create": (c_int, [c_i64, c_vp, c_i64, c_vp, ctypes.POINTER(c_vp)]),
    "ctn_gemm_grouped_plan_flops": (c_dbl, [c_vp]),
    "ctn_gemm_grouped_f64": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "ctn_gemm_grouped_plan_destroy": (None, [c_vp]),
    "ctn_split_gemm_workspace_bytes": (c_size, [c_i64, c_i64, c_i64, c_int]),
    "ctn_split_gemm_f64": (c_int, [c_i64, c_i64, c_i64, c_vp, c_vp, c_vp, c_int, c_vp, c_vp]),
    "ctn_split_gemm_f64_noalloc": (c_int, [c_i64, c_i64, c_i64, c_vp, c_vp, c_vp, c_int, c_vp]),
    "ctn_selftest_wait_timeout": (c_int, [c_int, ctypes.c_longlong, c_vp]),
    "ctn_selftest_barrier_timeout": (c_int, [ctypes.c_longlong, c_vp]),
    "ctn_dot_f64": (c_int, [c_vp, c_vp, c_i64, c_vp, c_vp]),
    "ctn_nrm2_f64": (c_int, [c_vp, c_i64, c_vp, c_vp]),
    "ctn_axpy_f64": (c_int, [c_vp, c_vp, c_i64, c_vp, c_dbl, c_vp]),
    "ctn_scal_f64": (c_int, [c_vp, c_i64, c_vp, c_int, c_vp]),
    "ctn_tridiag_eigh": (c_int, [c_int, P_dbl, P_dbl, P_dbl, P_dbl]),
    "ctn_heff2_plan_create": (c_int, [ctypes.POINTER(Heff2Desc), ctypes.POINTER(c_vp)]),
    "ctn_heff2_flops": (c_dbl, [c_vp]),
    "ctn_heff2_psi_elems": (c_size, [c_vp]),
    "ctn_heff2_workspace_bytes": (c_size, [c_vp, c_int]),
    "ctn_heff2_set_env": (c_int, [c_vp, c_vp, c_vp, c_vp, c_int, c_vp]),
    "ctn_heff2_matvec": (c_int, [c_vp, c_vp, c_vp, c_int, c_vp]),
    "ctn_heff2_plan_destroy": (None, [c_vp]),
    "ctn_heff2_set_tiles": (c_int, [c_vp, c_int, c_int, c_int]),
    "ctn_heff2_set_epilogue": (c_int, [c_vp, c_int, c_int, c_int]),
    "ctn_heff2_profile": (c_int, [c_vp, c_vp, c_vp, c_int, c_int, P_dbl, ctypes.POINTER(c_int), c_vp]),
    "ctn_heff2_gemm_flops": (c_dbl, [c_vp, c_int]),
    "ctn_heff2_split_gemm_flops": (c_dbl, [c_vp, c_int, c_int]),
    "ctn_heff2_split_stats": (c_int, [c_vp, c_int, ctypes.POINTER(c_dbl)]),
    "ctn_heff2_batch_create": (c_int, [ctypes.POINTER(c_vp), c_int, P_i64, P_i64, P_i64, c_int, c_int, c_int, c_int,
                                       ctypes.POINTER(c_vp)]),
    "ctn_heff2_batch_workspace_bytes": (c_size, [c_vp]),
    "ctn_heff2_batch_gemm_flops": (c_dbl, [c_vp]),
    "ctn_heff2_batch_stats": (c_int, [c_vp, ctypes.POINTER(c_dbl)]),
    "ctn_heff2_batch_set_env": (c_int, [c_vp, c_vp, c_vp, c_vp, c_vp]),
    "ctn_heff2_batch_matvec": (c_int, [c_vp, c_vp, c_vp, c_vp]),
    "ctn_heff2_batch_profile": (c_int, [c_vp, c_vp, c_vp, c_int, P_dbl, c_vp]),
    "ctn_heff2_batch_destroy": (None, [c_vp]),
    "ctn_lanczos_gnd": (c_int, [MATVEC_FN, c_vp, c_vp, c_i64, c_int, c_dbl, c_vp, c_vp, c_vp, P_dbl,
                                ctypes.POINTER(c_int), c_vp]),
    "ctn_lanczos_refined": (c_int, [MATVEC_FN, c_vp, MATVEC_FN, c_vp, c_vp, c_i64, c_int, c_int, c_dbl, c_vp, c_vp,
                                    c_vp, P_dbl, P_dbl, ctypes.POINTER(c_int), P_i64, c_vp]),
    "ctn_lanczos_exp_work_doubles": (c_size, [c_i64, c_int]),
    "ctn_lanczos_exp": (c_int, [MATVEC_FN, c_vp, c_vp, c_i64, c_dbl, c_dbl, c_dbl, c_int, c_vp, c_vp, c_vp, c_vp,
                                ctypes.POINTER(c_int), c_vp]),
    "ctn_lanczos_which_work_doubles": (c_size, [c_i64, c_int]),
    "ctn_lanczos_which": (c_int, [MATVEC_FN, c_vp, c_vp, c_i64, c_int, c_int, c_int, c_int, c_dbl, c_vp, c_vp, P_dbl,
                                  c_vp, ctypes.POINTER(c_int), ctypes.POINTER(c_int), c_vp]),
    "ctn_sym_eigh": (c_int, [c_int, P_dbl, P_dbl, P_dbl]),
    "ctn_heff2_lanczos_refined": (c_int, [c_vp, c_int, c_vp, c_int, c_int, c_dbl, c_vp, c_vp, c_vp, P_dbl, P_dbl,
                                          ctypes.POINTER(c_int), P_i64, c_vp]),
    "ctn_heff2_lanczos_gnd": (c_int, [c_vp, c_int, c_vp, c_int, c_dbl, c_vp, c_vp, c_vp, P_dbl,
                                      ctypes.POINTER(c_int), c_vp]),
}

_lib = None


def lib():
    """Load the library once; raises CytnxError when it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise CytnxError(f"{LIB_PATH} is missing: build it with `python -m cytnx_b200.build`")
        l = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(l, name)
            fn.restype = res
            fn.argtypes = args
        _lib = l
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(status: int, what: str = "") -> None:
    if status != 0:
        msg = lib().ctn_last_error().decode(errors="replace")
        raise CytnxError(f"[ERROR]{'[' + what + ']' if what else ''} {msg} (status {status})")


def stream_ptr(stream=None) -> int:
    """Raw cudaStream_t of a torch stream (default: the current stream)."""
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)
