"""Split-precision tcgen05 GEMM (3xTF32, BF16x3) against an FP64 reference product."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

# Relative Frobenius-norm error bounds of the split forms.  3xTF32 keeps ~22 significant
# bits per operand (x = hi + lo, dropped lo*lo term ~2^-22 relative) and accumulates in
# the tensor core's FP32, whose rounding error grows like sqrt(K) * 2^-24 relative to the
# result: bound 1e-6 + 2e-7*sqrt(K).  BF16x3 keeps ~16 bits per operand: 5e-4.
def tol(prec, K):
    return 1e-6 + 2e-7 * K ** 0.5 if prec == "3xtf32" else 5e-4


def split_gemm(A, B, prec):
    from cytnx_b200 import _lib

    p = _lib.PRECISIONS[prec]
    M, K = A.shape
    N = B.shape[1]
    ws = torch.empty(_lib.lib().ctn_split_gemm_workspace_bytes(M, N, K, p), dtype=torch.uint8, device="cuda")
    C = torch.empty(M, N, dtype=torch.float64, device="cuda")
    _lib.check(_lib.lib().ctn_split_gemm_f64(M, N, K, A.data_ptr(), B.data_ptr(), C.data_ptr(), p,
                                             ws.data_ptr(), _lib.stream_ptr()), "split_gemm")
    return C


@pytest.mark.parametrize("prec", ["3xtf32", "bf16x3"])
@pytest.mark.parametrize("shape", [(128, 128, 32), (128, 128, 256), (300, 200, 100), (1000, 700, 513), (7, 5, 3)])
def test_split_gemm_dense(prec, shape):
    M, N, K = shape
    g = torch.Generator(device="cuda").manual_seed(M * 7 + N)
    A = torch.randn(M, K, dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn(K, N, dtype=torch.float64, device="cuda", generator=g)
    C = split_gemm(A, B, prec)
    ref = A @ B
    err = (torch.linalg.matrix_norm(C - ref) / torch.linalg.matrix_norm(ref)).item()
    assert err < tol(prec, K), err
    # twice in a row (ring phases and accumulator reuse)
    C2 = split_gemm(A, B, prec)
    assert torch.equal(C, C2)


def _heff(D, seed=0):
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    spec = W.xxz_spec(D)
    psi, L, M1, M2, R = W.build_two_site(spec, W.xxz_mpo_values(), seed=seed, device=0)
    return psi, c.TwoSiteHeff(L, M1, M2, R, psi)


@pytest.mark.parametrize("prec,bound", [("3xtf32", 1e-5), ("bf16x3", 2e-3)])
@pytest.mark.parametrize("D", [24, 256, 1024])
def test_heff_split_matches_fp64(prec, bound, D):
    """Split-precision H_eff matvec vs the FP64 path (itself checked against the oracle)."""
    psi, H = _heff(D, seed=4)
    x = psi.flat_view()
    y64 = torch.empty_like(x)
    ys = torch.empty_like(x)
    H.apply_flat(x, y64, "fp64")
    H.apply_flat(x, ys, prec)
    err = (torch.linalg.vector_norm(ys - y64) / torch.linalg.vector_norm(y64)).item()
    assert err < bound, err
    ys2 = torch.empty_like(x)
    H.apply_flat(x, ys2, prec)  # deterministic: same bits on a second call
    assert torch.equal(ys, ys2)


def test_heff_split_random_vectors_linear():
    psi, H = _heff(256, seed=5)
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.randn(H.n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(H.n, dtype=torch.float64, device="cuda", generator=g)
    hx, hy, hz = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    H.apply_flat(x, hx, "3xtf32")
    H.apply_flat(y, hy, "3xtf32")
    H.apply_flat(x + y, hz, "3xtf32")
    lin = (torch.linalg.vector_norm(hz - hx - hy) / torch.linalg.vector_norm(hz)).item()
    assert lin < 1e-5


@pytest.mark.parametrize("prec", ["3xtf32", "bf16x3"])
def test_heff_split_tile_widths_agree(prec):
    """Every compiled tile width gives the same matvec (to the split tolerance)."""
    psi, H = _heff(512, seed=8)
    x = psi.flat_view()
    y64 = torch.empty_like(x)
    H.apply_flat(x, y64, "fp64")
    for b1, b4 in [(64, 96), (128, 144), (160, 160), (192, 256), (256, 64)]:
        H.set_tiles(b1, b4, prec)
        y = torch.empty_like(x)
        H.apply_flat(x, y, prec)
        err = (torch.linalg.vector_norm(y - y64) / torch.linalg.vector_norm(y64)).item()
        assert err < (1e-5 if prec == "3xtf32" else 2e-3), (b1, b4, err)
    tuned = H.autotune(prec, reps=2)
    # any of the default candidates (1-CTA widths and one 2-CTA width per step)
    assert tuned["step1"] in (128, 160, 192, 256, -192) and tuned["step4"] in (96, 128, 144, 160, 256, -128)
    assert tuned["epilogue"][0] in (0, 1, 2) and tuned["epilogue"][1] in (0, 1, 2)


@pytest.mark.parametrize("prec", ["3xtf32", "bf16x3"])
def test_heff_split_pair_tiles_match_single_cta(prec):
    """2-CTA (cta_group::2, 256-row) tiles give the 1-CTA result: same products, same
    K order; the FP32 accumulators agree to rounding."""
    psi, H = _heff(512, seed=9)
    x = psi.flat_view()
    y64 = torch.empty_like(x)
    H.apply_flat(x, y64, "fp64")
    H.set_tiles(128, 128, prec)
    y1 = torch.empty_like(x)
    H.apply_flat(x, y1, prec)
    for b1, b4 in [(-128, -128), (-256, -192), (-192, -256), (-128, 128), (160, -128)]:
        H.set_tiles(b1, b4, prec)
        y = torch.empty_like(x)
        H.apply_flat(x, y, prec)
        d = (torch.linalg.vector_norm(y - y1) / torch.linalg.vector_norm(y1)).item()
        e = (torch.linalg.vector_norm(y - y64) / torch.linalg.vector_norm(y64)).item()
        assert d < 1e-6 and e < 2e-5, (b1, b4, d, e)


@pytest.mark.parametrize("prec", ["3xtf32", "bf16x3"])
def test_epilogue_forms_are_bitwise_equal(prec):
    """The direct, the shared-memory-staged and the TMEM-fragment epilogues store the same
    accumulators (tile widths that are not multiples of 32 included: a fragment reaching past
    the tile edge must not write the next tile's columns)."""
    from cytnx_b200 import _lib

    psi, H = _heff(384, seed=10)
    x = psi.flat_view()
    H.set_tiles(160, 144, prec)
    out = []
    for e1, e4 in [(0, 0), (1, 1), (0, 1), (-1, -1), (2, 2), (2, 0), (1, 2)]:
        _lib.check(_lib.lib().ctn_heff2_set_epilogue(H._h, _lib.PRECISIONS[prec], e1, e4))
        y = torch.zeros_like(x)
        H.apply_flat(x, y, prec)
        out.append(y)
    for y in out[1:]:
        assert torch.equal(y, out[0])
    for b1, b4 in [(48, 96), (256, 128), (-128, 128)]:  # and other widths (2-CTA: 2 runs as staged)
        H.set_tiles(b1, b4, prec)
        ys = []
        for e in (1, 2):
            _lib.check(_lib.lib().ctn_heff2_set_epilogue(H._h, _lib.PRECISIONS[prec], e, e))
            y = torch.zeros_like(x)
            H.apply_flat(x, y, prec)
            ys.append(y)
        assert torch.equal(ys[0], ys[1]), (b1, b4)
