"""The CPU oracle against the reference's own golden fixtures (no GPU)."""
import itertools

import numpy as np
import pytest

import oracle as O
from conftest import golden_oracle_tensor, load_golden


@pytest.mark.parametrize("case,labels", [(1, (["a", "b"], ["b", "c"])), (2, (["a", "b"], ["b", "c"])),
                                         (3, (["a", "b", "c"], ["c", "d", "e"]))])
def test_block_contract_golden(case, labels):
    # tests/BlockUniTensor_test.cpp:679-717 (tolerance there: 1e-5)
    L = golden_oracle_tensor(f"block_contract_L{case}", labels[0])
    R = golden_oracle_tensor(f"block_contract_R{case}", labels[1])
    A = golden_oracle_tensor(f"block_contract_ans{case}")
    out = L.contract(R)
    assert np.array_equal(out.itoi, A.itoi)
    assert len(out.blocks) == len(A.blocks)
    for o, a in zip(out.blocks, A.blocks):
        np.testing.assert_allclose(o, a, rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["block_contract_L1", "block_contract_L3", "block_contract_R3",
                                  "block_contract_ans3", "block_permute_T1", "block_permute_ans1"])
def test_block_enumeration_golden(name):
    # BlockUniTensor::Init order is what the saved files hold
    t = golden_oracle_tensor(name)
    assert np.array_equal(O.enumerate_blocks(t.bonds), t.itoi)


@pytest.mark.parametrize("case,mapper", [(1, [1, 2, 0]), (2, [1, 0]), (3, [1, 0])])
def test_block_permute_golden(case, mapper):
    # tests/BlockUniTensor_test.cpp:308-360 (exact)
    T = golden_oracle_tensor(f"block_permute_T{case}")
    A = golden_oracle_tensor(f"block_permute_ans{case}")
    assert np.array_equal(T.permute(mapper).dense(), A.dense())


def test_dense_contract_golden():
    # tests/DenseUniTensor_test.cpp:2594-2619: ut1 (a,b,c,d) x ut2 with 1, 2, 3 shared labels
    u1 = load_golden("dense_denseutensor1")["block"]
    u2 = load_golden("dense_denseutensor2")["block"]
    for k in (1, 2, 3):
        ans = load_golden(f"dense_densecontres{k}")["block"]
        out = O.tensordot(u1, u2, list(range(k)), list(range(k)))
        np.testing.assert_allclose(out, ans, rtol=0, atol=1e-10)


def test_permute_matches_numpy_all_rank4():
    rng = np.random.default_rng(0)
    a = rng.standard_normal((6, 2, 3, 5))
    for p in itertools.permutations(range(4)):
        assert np.array_equal(O.permute(a, p), a.transpose(p))


def test_permute_meta_rules():
    # Tensor_impl::permute composes mappers (src/backend/Tensor_impl.cpp:38-86)
    shape, mapper, inv = [2, 3, 4], [0, 1, 2], [0, 1, 2]
    s1, m1, i1, c1 = O.permute_meta(shape, mapper, inv, [2, 0, 1])
    assert s1 == [4, 2, 3] and m1 == [2, 0, 1] and not c1
    s2, m2, i2, c2 = O.permute_meta(s1, m1, i1, [1, 2, 0])
    assert s2 == [2, 3, 4] and m2 == [0, 1, 2] and c2


def test_lanczos_blocks_golden():
    # tests/linalg_test/Lanczos_Gnd_test.cpp:392-422: block H from lan_block_{A,B,C}; E vs Eigh to 1e-12
    z = load_golden("lanczos_blocks")
    blocks = [z[k] for k in "ABC"]
    H = np.zeros((27, 27))
    for i, b in enumerate(blocks):
        H[9 * i:9 * i + 9, 9 * i:9 * i + 9] = b
    E0 = np.linalg.eigvalsh(H).min()
    rng = np.random.default_rng(1)
    x0 = rng.standard_normal(27)
    E, v, it = O.lanczos_gnd_ut(lambda x: H @ x, x0, 1e-15, 10000)
    assert abs(E - E0) < 1e-12
    assert np.linalg.norm(H @ v - E * v) < 1e-6


def test_lanczos_arange_golden():
    # tests/linalg_test/Lanczos_Gnd_test.cpp:377-390: A = arange(27*27); H = A + A^T; E = -1628.9964650426593
    A = np.arange(27 * 27, dtype=np.float64).reshape(27, 27)
    H = A + A.T
    E, v, it = O.lanczos_gnd_ut(lambda x: H @ x, np.arange(27.0), 1e-15, 10000)
    assert abs(E - (-1628.9964650426593)) < 1e-5


def test_dstev_matches_eigh():
    rng = np.random.default_rng(3)
    d, e = rng.standard_normal(12), rng.standard_normal(11)
    w, z = O.dstev(d, e)
    T = np.diag(d) + np.diag(e, 1) + np.diag(e, -1)
    np.testing.assert_allclose(w, np.linalg.eigvalsh(T), atol=1e-12)
    for j in range(12):
        np.testing.assert_allclose(T @ z[j], w[j] * z[j], atol=1e-10)
