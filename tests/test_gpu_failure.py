"""Fault injection on the device path without a GPU fault: NaN injected into an input vector
or an environment block comes back as an error status from the drivers, and the context stays
usable for the next call."""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _build(D=64, seed=1):
    from cytnx_b200 import workloads as W

    return W.build_two_site(W.xxz_spec(D), W.xxz_mpo_values(1.0, 1.0), seed=seed, device=0)


def test_nan_in_start_vector_is_reported():
    import cytnx_b200 as c
    from cytnx_b200._lib import CytnxError

    psi, L, M1, M2, R = _build()
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    bad = psi.clone()
    bad.flat_view()[3] = math.nan
    with pytest.raises(CytnxError, match="non-finite"):
        H.lanczos_refined(bad, precision="bf16x3", krylov_dim=8, max_restarts=4)
    with pytest.raises(CytnxError, match="non-finite"):
        c.linalg.Lanczos(Hop=H, Tin=bad, method="Gnd", Maxiter=4, CvgCrit=1e-12)
    # the context is intact: the same operator still runs on a good vector
    r = H.lanczos_refined(psi, precision="bf16x3", krylov_dim=8, max_restarts=40, tol=1e-10)
    assert math.isfinite(r["energy"]) and r["residual"] <= 1e-10 * abs(r["energy"])


def test_nan_in_environment_is_reported():
    import cytnx_b200 as c
    from cytnx_b200._lib import CytnxError

    psi, L, M1, M2, R = _build(seed=2)
    Lb = L.clone()
    Lb.flat_view()[0] = math.nan
    H = c.TwoSiteHeff(Lb, M1, M2, R, psi)
    with pytest.raises(CytnxError, match="non-finite"):
        H.lanczos_refined(psi, precision="bf16x3", krylov_dim=8, max_restarts=4)
    H2 = c.TwoSiteHeff(L, M1, M2, R, psi)
    x = psi.flat_view()
    y = torch.empty_like(x)
    H2.apply_flat(x, y, "fp64")
    assert torch.isfinite(y).all()


def test_krylov_grid_barrier_expires_and_context_survives():
    """The fused Krylov step's grid barrier (ctn_selftest_barrier_timeout: a barrier that waits
    for one arrival more than the grid has, 2^12 probes per CTA): every CTA's wait runs out,
    the host sees CTN_ERR_TIMEOUT, and a refined Lanczos run on the same context, whose Krylov
    steps use the same kernel, still converges."""
    import cytnx_b200 as c
    from cytnx_b200 import _lib

    lib = _lib.lib()
    rc = lib.ctn_selftest_barrier_timeout(1 << 12, _lib.stream_ptr())
    assert rc == 4, (rc, lib.ctn_last_error())
    assert b"bounded wait expired" in lib.ctn_last_error()
    psi, L, M1, M2, R = _build(seed=5)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    r = H.lanczos_refined(psi, precision="bf16x3", krylov_dim=8, max_restarts=40, tol=1e-10)
    assert math.isfinite(r["energy"]) and r["residual"] <= 1e-10 * abs(r["energy"])


@pytest.mark.parametrize("precision", [1, 2])
def test_tcgen05_bounded_wait_expires_and_context_survives(precision):
    """The tcgen05 GEMM's bounded waits (ctn_selftest_wait_timeout: a producer that issues no
    copies, 2^16 probes per wait): the MMA warp's first wait runs out, the kernel records
    the error, stops its other roles, frees TMEM and returns; the host sees CTN_ERR_TIMEOUT
    and the next GEMM on the same context is correct."""
    from cytnx_b200 import _lib

    lib = _lib.lib()
    rc = lib.ctn_selftest_wait_timeout(precision, 1 << 16, _lib.stream_ptr())
    assert rc == 4, (rc, lib.ctn_last_error())
    assert b"bounded wait expired" in lib.ctn_last_error()
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(300, 200, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(200, 150, dtype=torch.float64, device="cuda", generator=g)
    ws = torch.empty(lib.ctn_split_gemm_workspace_bytes(300, 150, 200, precision), dtype=torch.uint8, device="cuda")
    C = torch.empty(300, 150, dtype=torch.float64, device="cuda")
    _lib.check(lib.ctn_split_gemm_f64(300, 150, 200, A.data_ptr(), B.data_ptr(), C.data_ptr(), precision,
                                      ws.data_ptr(), _lib.stream_ptr()), "split_gemm")
    ref = A @ B
    assert (torch.linalg.matrix_norm(C - ref) / torch.linalg.matrix_norm(ref)).item() < 1e-4
