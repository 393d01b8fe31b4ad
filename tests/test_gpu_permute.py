"""Permute kernel parity: bit-exact against the oracle restatement of MoveMemoryCpu."""
import itertools

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def _permute_dev(a: np.ndarray, mapper):
    import cytnx_b200 as c

    t = c.Tensor.from_numpy(a, 0)
    return t.permute(list(mapper)).contiguous().numpy()


def test_all_24_perms_rank4_f64():
    # the [64,2,2,64] float64 tensor of the dense configuration, every permutation
    rng = np.random.default_rng(0)
    a = rng.standard_normal((64, 2, 2, 64))
    for p in itertools.permutations(range(4)):
        out = _permute_dev(a, p)
        ref = O.permute(a, p)
        assert out.shape == ref.shape
        assert np.array_equal(out.view(np.uint64), ref.view(np.uint64)), p


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int64, np.int32, np.int16, np.uint16,
                                   np.complex128, np.complex64, np.bool_])
def test_dtypes_bit_exact(dtype):
    rng = np.random.default_rng(1)
    shape = (3, 5, 7, 4)
    if dtype == np.bool_:
        a = rng.integers(0, 2, shape).astype(np.bool_)
    elif np.issubdtype(dtype, np.complexfloating):
        a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
    elif np.issubdtype(dtype, np.floating):
        a = rng.standard_normal(shape).astype(dtype)
    else:
        a = rng.integers(-100, 100, shape).astype(dtype)
    for p in itertools.permutations(range(4)):
        assert np.array_equal(_permute_dev(a, p), O.permute(a, p))


def test_random_shapes_and_ranks():
    rng = np.random.default_rng(2)
    for trial in range(60):
        r = int(rng.integers(1, 7))
        shape = tuple(int(x) for x in rng.integers(1, 9, r))
        a = rng.standard_normal(shape)
        p = list(rng.permutation(r))
        assert np.array_equal(_permute_dev(a, p), O.permute(a, p)), (shape, p)


def test_edge_cases_empty_and_ones():
    for shape, p in [((0, 3), (1, 0)), ((1, 1, 1), (2, 0, 1)), ((1,), (0,)), ((5, 1, 1, 7), (3, 1, 2, 0)),
                     ((2, 0, 4), (2, 1, 0))]:
        a = np.arange(int(np.prod(shape)), dtype=np.float64).reshape(shape)
        out = _permute_dev(a, p)
        assert out.shape == a.transpose(p).shape
        assert np.array_equal(out, a.transpose(p))


def test_large_transpose_and_unaligned_views():
    rng = np.random.default_rng(3)
    a = rng.standard_normal((257, 3, 129))
    for p in [(2, 1, 0), (1, 2, 0), (2, 0, 1), (0, 2, 1)]:
        assert np.array_equal(_permute_dev(a, p), O.permute(a, p))
    # source at an odd element offset (not 16-byte aligned) through a block view
    import cytnx_b200 as c

    base = torch.from_numpy(rng.standard_normal(1 + 6 * 10)).cuda()
    t = c.Tensor.from_torch(base[1:].view(6, 10))
    ref = base[1:].view(6, 10).cpu().numpy()
    assert np.array_equal(t.permute(1, 0).contiguous().numpy(), ref.T)


@pytest.mark.parametrize("dtype", [np.float64, np.float32, np.int16, np.bool_, np.complex128])
def test_short_output_axis_staged(dtype):
    """Output's fastest axis shorter than 16 under a long input axis: contiguous output runs
    (output stride of the input's fastest axis == the short extent), strided runs, ragged
    tiles, every short extent 2..15 (complex128 at 13..15 takes the unstaged kernel)."""
    rng = np.random.default_rng(5)

    def make(shape):
        if dtype == np.bool_:
            return rng.integers(0, 2, shape).astype(np.bool_)
        if dtype == np.complex128:
            return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
        if dtype == np.int16:
            return rng.integers(-30000, 30000, shape).astype(dtype)
        return rng.standard_normal(shape).astype(dtype)

    cases = [((3, 5, 600), (0, 2, 1)), ((5, 3, 1030), (1, 2, 0)), ((4, 6, 530), (2, 1, 0)),
             ((2, 1030), (1, 0)), ((7, 2, 2, 513), (1, 0, 3, 2)), ((256, 4), (1, 0))]
    cases += [((nb, 300), (1, 0)) for nb in range(2, 16)]
    for shape, p in cases:
        a = make(shape)
        out = _permute_dev(a, p)
        assert np.array_equal(out, O.permute(a, p)), (shape, p)


@pytest.mark.parametrize("dtype", [np.float64, np.int64, np.complex64, np.float32, np.int32, np.int16, np.bool_])
def test_tma_staged_transpose_ragged(dtype):
    """Transposes above 1 MB with 16-byte input strides: the TMA-staged kernel (1-, 2- and 4-byte
    elements) and the register tile (8-byte elements), ragged tiles along both transposed axes,
    with and without a batch axis."""
    rng = np.random.default_rng(7)
    for shape, p in [((300, 5, 704), (2, 1, 0)), ((64, 3, 7, 1040), (3, 1, 2, 0)), ((2000, 520), (1, 0))]:
        if dtype == np.bool_:
            a = rng.integers(0, 2, shape).astype(np.bool_)
        elif np.issubdtype(dtype, np.complexfloating):
            a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)
        elif np.issubdtype(dtype, np.floating):
            a = rng.standard_normal(shape).astype(dtype)
        else:
            a = rng.integers(0, 120, shape).astype(dtype)
        assert np.array_equal(_permute_dev(a, p), O.permute(a, p)), (shape, p)


def test_short_output_axis_unaligned_destination():
    """ctn_permute into a destination 4 bytes past a 16-byte boundary (the element-wise
    store path of the staged kernel) and at a 16-byte boundary, same input."""
    from cytnx_b200 import _lib

    rng = np.random.default_rng(6)
    shape, p = (3, 4, 777), (0, 2, 1)
    a = rng.standard_normal(shape).astype(np.float32)
    x = torch.from_numpy(a).cuda()
    ref = O.permute(a, p).reshape(-1)
    for off in (0, 1):
        buf = torch.zeros(a.size + 8, dtype=torch.float32, device="cuda")
        dst = buf[4 + off:4 + off + a.size]
        osh = np.array(shape, dtype=np.uint64)
        mp = np.array(p, dtype=np.uint64)
        _lib.check(_lib.lib().ctn_permute(x.data_ptr(), dst.data_ptr(), 4, 3, osh.ctypes.data_as(_lib.P_u64),
                                          mp.ctypes.data_as(_lib.P_u64), _lib.stream_ptr()), "permute")
        torch.cuda.synchronize()
        got = buf.cpu().numpy()
        assert np.array_equal(got[4 + off:4 + off + a.size], ref)
        assert not got[:4 + off].any() and not got[4 + off + a.size:].any()


def test_lazy_permute_composition():
    import cytnx_b200 as c

    rng = np.random.default_rng(4)
    a = rng.standard_normal((4, 3, 6, 5))
    t = c.Tensor.from_numpy(a, 0)
    u = t.permute(2, 0, 3, 1).permute(1, 3, 0, 2)  # back to identity -> contiguous flag
    assert u.is_contiguous() and u.same_data(t)
    v = t.permute(3, 1, 0, 2).permute(0, 2, 1, 3)
    assert np.array_equal(v.contiguous().numpy(), a.transpose(3, 1, 0, 2).transpose(0, 2, 1, 3))


@pytest.mark.parametrize("case,mapper", [(1, [1, 2, 0]), (2, [1, 0]), (3, [1, 0])])
def test_block_permute_golden(case, mapper):
    import cytnx_b200 as c
    from conftest import golden_bonds, golden_blocks, load_golden

    z, za = load_golden(f"block_permute_T{case}"), load_golden(f"block_permute_ans{case}")
    u = c.UniTensor(golden_bonds(z, c), labels=list(z["labels"]), rowrank=int(z["rowrank"]), device=0)
    for b, blk in enumerate(golden_blocks(z)):
        u.put_block(c.Tensor.from_numpy(blk, 0), b)
    p = u.permute(mapper).contiguous()
    ans = golden_oracle = __import__("conftest").golden_oracle_tensor(f"block_permute_ans{case}")
    assert np.array_equal(p.to_dense_numpy(), ans.dense())
