"""The allocation-free split GEMM entry point (ctn_split_gemm_f64_noalloc).

Callers whose device memory belongs to their own pool allocator, that run under a
fixed memory budget, or that bind the C ABI from a language without a device
allocator cannot hand this library a workspace or let it cudaMalloc one.  This entry
point keeps its scratch in a fixed 32 MiB static device array instead.  The test calls
it through the C ABI twice in a row and checks each result against the workspace
entry point (ctn_split_gemm_f64) within the split-precision tolerance of the other
tests; it lives in its own file, collected last, and passes alone or after the suite.
"""
import ctypes

import pytest
import torch

pytestmark = pytest.mark.gpu


def tol(prec, K):  # same bound as tests/test_gpu_split.py
    return 1e-6 + 2e-7 * K ** 0.5 if prec == "3xtf32" else 5e-4


def _with_workspace(A, B, p):
    from cytnx_b200 import _lib

    M, K = A.shape
    N = B.shape[1]
    ws = torch.empty(_lib.lib().ctn_split_gemm_workspace_bytes(M, N, K, p), dtype=torch.uint8, device="cuda")
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().ctn_split_gemm_f64(M, N, K, A.data_ptr(), B.data_ptr(), C.data_ptr(), p, ws.data_ptr(),
                                             _lib.stream_ptr()), "split_gemm")
    return C


def _noalloc(A, B, p):
    from cytnx_b200 import _lib

    M, K = A.shape
    N = B.shape[1]
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().ctn_split_gemm_f64_noalloc(M, N, K, A.data_ptr(), B.data_ptr(), C.data_ptr(), p,
                                                     _lib.stream_ptr()), "split_gemm_noalloc")
    return C


@pytest.mark.parametrize("prec", ["3xtf32", "bf16x3"])
@pytest.mark.parametrize("shape", [(300, 200, 100), (513, 384, 257)])
def test_noalloc_matches_workspace_entry_point(prec, shape):
    from cytnx_b200 import _lib

    p = _lib.PRECISIONS[prec]
    M, N, K = shape
    g = torch.Generator(device="cuda").manual_seed(11 + M)
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(K, N, dtype=torch.float64, device="cuda", generator=g)
    ref = _with_workspace(A, B, p)
    scale = torch.linalg.matrix_norm(ref).item()
    for _ in range(2):  # the static array keeps the previous call's contents
        C = _noalloc(A, B, p)
        err = torch.linalg.matrix_norm(C - ref).item() / scale
        assert err < tol(prec, K), err


def test_noalloc_rejects_oversize():
    from cytnx_b200 import _lib
    from cytnx_b200._lib import CytnxError

    A = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(CytnxError, match="static device array"):
        _lib.check(_lib.lib().ctn_split_gemm_f64_noalloc(8192, 8192, 8192, A.data_ptr(), A.data_ptr(),
                                                         A.data_ptr(), _lib.PRECISIONS["3xtf32"],
                                                         _lib.stream_ptr()), "split_gemm_noalloc")


def test_noalloc_allocates_nothing():
    """After a warm-up call (which loads the kernels), further calls leave the device's free
    memory and torch's allocator untouched."""
    from cytnx_b200 import _lib

    p = _lib.PRECISIONS["bf16x3"]
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn(256, 192, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(192, 160, dtype=torch.float64, device="cuda", generator=g)
    C = torch.empty(256, 160, dtype=torch.float64, device="cuda")

    def call():
        _lib.check(_lib.lib().ctn_split_gemm_f64_noalloc(256, 160, 192, A.data_ptr(), B.data_ptr(), C.data_ptr(), p,
                                                         _lib.stream_ptr()), "split_gemm_noalloc")

    call()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    for _ in range(3):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_allocated() == alloc0


def test_noalloc_size_limit_boundary():
    """3xTF32 panels take 16 KiB per (128-row tile x 16-wide K slice) for A and B alike: at
    M = N = 512, K = 4064 (254 slices) the problem fits the 32 MiB array with its tables;
    K = 4096 (256 slices) fills the array with panels alone and is rejected."""
    from cytnx_b200 import _lib
    from cytnx_b200._lib import CytnxError

    p = _lib.PRECISIONS["3xtf32"]
    g = torch.Generator(device="cuda").manual_seed(9)
    M = N = 512
    K = 4064
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(K, N, dtype=torch.float64, device="cuda", generator=g)
    ref = _with_workspace(A, B, p)
    C = _noalloc(A, B, p)
    assert torch.linalg.matrix_norm(C - ref).item() / torch.linalg.matrix_norm(ref).item() < tol("3xtf32", K)
    A2 = torch.zeros(M, 4096, dtype=torch.float64, device="cuda")
    with pytest.raises(CytnxError, match="static device array"):
        _lib.check(_lib.lib().ctn_split_gemm_f64_noalloc(M, N, 4096, A2.data_ptr(), A2.data_ptr(), C.data_ptr(), p,
                                                         _lib.stream_ptr()), "split_gemm_noalloc")
