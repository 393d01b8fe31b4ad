"""Block-sparse contraction parity against the oracle and the reference goldens."""
import numpy as np
import pytest
import torch

import oracle as O
from conftest import golden_bonds, golden_blocks, golden_oracle_tensor, load_golden

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative, FP64 vs the FP64 oracle (different summation order only)


def to_device(ot, c, part=None):
    """oracle.BlockTensor -> cytnx_b200 UniTensor (optionally the real or imag part)."""
    bonds = [c.Bond(b.type, b.qnums, b.degs, [c.Symmetry(s[0], s[1]) for s in b.syms]) for b in ot.bonds]
    u = c.UniTensor(bonds, labels=ot.labels, rowrank=ot.rowrank, device=0)
    idx = u._layout.index()
    for t, blk in zip(ot.itoi.tolist(), ot.blocks):
        x = blk.real if part == "re" else blk.imag if part == "im" else blk
        b = idx[tuple(t)]
        off = int(u._layout.offs[b])
        u._data[off: off + x.size] = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64).reshape(-1)).cuda()
    return u


def assert_close_blocks(u, ot, tol=TOL, part=None):
    assert np.array_equal(u._layout.itoi, ot.itoi)
    scale = max(1e-300, max((np.abs(b).max() for b in ot.blocks if b.size), default=1.0))
    for b, ref in enumerate(ot.blocks):
        r = ref.real if part == "re" else ref.imag if part == "im" else ref
        got = u.get_block_(b).numpy()
        assert got.shape == r.shape
        np.testing.assert_allclose(got, r, rtol=0, atol=tol * scale)


@pytest.mark.parametrize("case,labels", [(1, (["a", "b"], ["b", "c"])), (2, (["a", "b"], ["b", "c"]))])
def test_golden_contract_real(case, labels):
    import cytnx_b200 as c

    L = golden_oracle_tensor(f"block_contract_L{case}", labels[0])
    R = golden_oracle_tensor(f"block_contract_R{case}", labels[1])
    A = golden_oracle_tensor(f"block_contract_ans{case}")
    out = c.Contract(to_device(L, c), to_device(R, c))
    assert_close_blocks(out, A, 1e-12)


def test_golden_contract3_complex_by_parts():
    """Case 3 is complex128; the engine is real FP64, and contraction is bilinear:
    re(LR) = re L re R - im L im R, im(LR) = re L im R + im L re R."""
    import cytnx_b200 as c

    L = golden_oracle_tensor("block_contract_L3", ["a", "b", "c"])
    R = golden_oracle_tensor("block_contract_R3", ["c", "d", "e"])
    A = golden_oracle_tensor("block_contract_ans3")
    Lr, Li, Rr, Ri = to_device(L, c, "re"), to_device(L, c, "im"), to_device(R, c, "re"), to_device(R, c, "im")
    re = c.Contract(Lr, Rr) - c.Contract(Li, Ri)
    im = c.Contract(Lr, Ri) + c.Contract(Li, Rr)
    assert len(re._layout.itoi) == 96
    assert_close_blocks(re, A, 1e-12, "re")
    assert_close_blocks(im, A, 1e-12, "im")


def test_dense_contract_golden_by_parts():
    import cytnx_b200 as c

    u1 = load_golden("dense_denseutensor1")["block"]
    u2 = load_golden("dense_denseutensor2")["block"]
    for k in (1, 2, 3):
        ans = load_golden(f"dense_densecontres{k}")["block"]
        outs = []
        for a in (u1.real, u1.imag):
            for b in (u2.real, u2.imag):
                out = c.linalg.Tensordot(c.Tensor.from_numpy(np.ascontiguousarray(a), 0),
                                         c.Tensor.from_numpy(np.ascontiguousarray(b), 0),
                                         list(range(k)), list(range(k)))
                outs.append(out.numpy())
        got = (outs[0] - outs[3]) + 1j * (outs[1] + outs[2])
        np.testing.assert_allclose(got, ans, rtol=0, atol=1e-10 * np.abs(ans).max())


def _random_block(c, bonds_spec, labels, rng):
    ob = [O.Bond(t, q, d) for t, q, d in bonds_spec]
    ot = O.BlockTensor(ob, labels, 1)
    ot.blocks = [rng.standard_normal(b.shape) for b in ot.blocks]
    return ot, to_device(ot, c)


def test_random_contractions_with_lazy_permutes():
    import cytnx_b200 as c

    rng = np.random.default_rng(7)
    qa = (np.array([[-1], [0], [1], [2]]), np.array([3, 5, 4, 2]))
    qb = (np.array([[0], [1], [-1]]), np.array([2, 3, 2]))
    qc = (np.array([[-2], [0], [1], [2]]), np.array([4, 1, 6, 3]))
    for trial in range(6):
        A_o, A = _random_block(c, [(-1, *qa), (1, *qb), (1, *qc)], ["i", "j", "k"], rng)
        B_o, B = _random_block(c, [(-1, *qc), (-1, *qb), (1, *qa)], ["k", "j", "l"], rng)
        pa = list(rng.permutation(3))
        pb = list(rng.permutation(3))
        A_p, B_p = A.permute(pa), B.permute(pb)            # lazy on the device side
        A_op, B_op = A_o.permute(pa), B_o.permute(pb)      # materialised in the oracle
        out = c.Contract(A_p, B_p)
        ref = A_op.contract(B_op)
        assert out.labels() == ref.labels
        assert_close_blocks(out.contiguous(), ref)


def test_contract_rank4_two_common_legs_and_empty_blocks():
    import cytnx_b200 as c

    rng = np.random.default_rng(8)
    q1 = (np.array([[0], [1], [3]]), np.array([2, 3, 1]))   # charge 3 has no partner below
    q2 = (np.array([[0], [1]]), np.array([3, 2]))
    A_o, A = _random_block(c, [(-1, *q1), (-1, *q2), (1, *q2), (1, *q1)], ["a", "b", "c", "d"], rng)
    B_o, B = _random_block(c, [(-1, *q2), (-1, *q1), (1, *q2), (1, *q1)], ["c", "d", "e", "f"], rng)
    out = c.Contract(A, B)
    ref = A_o.contract(B_o)
    assert_close_blocks(out, ref)


def test_contract_errors():
    import cytnx_b200 as c

    rng = np.random.default_rng(9)
    q = (np.array([[0], [1]]), np.array([2, 2]))
    _, A = _random_block(c, [(-1, *q), (1, *q)], ["a", "b"], rng)
    _, B = _random_block(c, [(1, *q), (1, *q)], ["b", "c"], rng)  # b is BRA on both sides
    with pytest.raises(c.CytnxError):
        c.Contract(A, B)


TASK_DT = np.dtype([("c_off", "<i8"), ("m", "<i4"), ("n", "<i4"), ("ldc", "<i4"), ("pair_begin", "<i4"),
                    ("pair_count", "<i4"), ("pad_", "<i4")])
PAIR_DT = np.dtype([("a_off", "<i8"), ("b_off", "<i8"), ("k", "<i4"), ("lda", "<i4"), ("ldb", "<i4"),
                    ("flags", "<i4")])


@pytest.mark.parametrize("flags", [0, 1, 2, 3])
@pytest.mark.parametrize("shapes", ["wide", "narrow"])
def test_grouped_gemm_tile_widths(flags, shapes):
    """ctn_gemm_grouped_f64 (the Gemm_Batch replacement) against FP64 torch matmuls.  'wide':
    four 1024 x 1024 tasks (1024 tiles of 64 x 64, above six per SM: the 64-wide kernel);
    'narrow': ragged small tasks (the 64 x 32 kernel).  Two pairs per task with k not a
    multiple of 16, every operand orientation, one task without pairs (zeros)."""
    import ctypes

    from cytnx_b200 import _lib

    g = torch.Generator().manual_seed(11 + flags)
    if shapes == "wide":
        mn = [(1024, 1024)] * 4
    else:
        mn = [(70, 70), (130, 6), (5, 200), (64, 33), (1, 1)]
    ks = [40, 23]
    a_parts, b_parts, tasks, pairs, refs = [], [], [], [], []
    a_off = b_off = c_off = 0
    for t, (m, n) in enumerate(mn):
        ref = torch.zeros(m, n, dtype=torch.float64)
        pb = len(pairs)
        npair = 0 if t == 2 else len(ks)
        for k in ks[:npair]:
            A = torch.randn(m, k, generator=g, dtype=torch.float64)
            B = torch.randn(k, n, generator=g, dtype=torch.float64)
            ref += A @ B
            As = A.t().contiguous() if flags & 1 else A
            Bs = B.t().contiguous() if flags & 2 else B
            pairs.append((a_off, b_off, k, m if flags & 1 else k, k if flags & 2 else n, flags))
            a_parts.append(As.reshape(-1))
            b_parts.append(Bs.reshape(-1))
            a_off += As.numel()
            b_off += Bs.numel()
        tasks.append((c_off, m, n, n, pb, npair, 0))
        refs.append((c_off, ref))
        c_off += m * n
    ta = np.array(tasks, dtype=TASK_DT)
    pa = np.array(pairs, dtype=PAIR_DT)
    A = torch.cat(a_parts).cuda()
    B = torch.cat(b_parts).cuda()
    C = torch.full((c_off,), float("nan"), dtype=torch.float64, device="cuda")
    plan = ctypes.c_void_p()
    _lib.check(_lib.lib().ctn_gemm_grouped_plan_create(len(ta), ta.ctypes.data, len(pa), pa.ctypes.data,
                                                       ctypes.byref(plan)), "plan")
    try:
        _lib.check(_lib.lib().ctn_gemm_grouped_f64(plan, A.data_ptr(), B.data_ptr(), C.data_ptr(), _lib.stream_ptr()),
                   "gemm")
        torch.cuda.synchronize()
    finally:
        _lib.lib().ctn_gemm_grouped_plan_destroy(plan)
    Ch = C.cpu()
    for off, ref in refs:
        got = Ch[off:off + ref.numel()].view(ref.shape)
        assert torch.allclose(got, ref, rtol=1e-12, atol=1e-12), (shapes, flags, float((got - ref).abs().max()))
