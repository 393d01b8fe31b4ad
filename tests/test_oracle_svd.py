"""The oracle's block SVD / truncation (oracle/svd.py) pinned to the reference's own fixtures:
Svd_truncate1 -> S_truncate1 (tests/linalg_test/linalg_test.cpp:57-67, to 1e-5) and
sym_UT_U1_exp_Svals_F64 with keepdim 5, with and without min_blockdim {1,1,0,2,0}
(tests/linalg_test/Gesvd_truncate_test.cpp:107-135: singular values to 1e-14 relative to
max(1, |S|), U S vT against the reconstructed tensor to 1e-14)."""
import numpy as np
import pytest

import oracle as O
from oracle import svd as OS
from conftest import golden_oracle_tensor, load_golden


def _ans_sectors(name):
    z = load_golden(name)
    q = z["bond0_qnums"].reshape(-1)
    vals = []
    pos = 0
    for shp in z["block_shapes"]:
        n = int(np.prod(shp))
        vals.append(z["data"][pos:pos + n])
        pos += n
    return [int(x) for x in q], vals


def test_svd_truncate1_matches_reference_singular_values():
    T = golden_oracle_tensor("svd_truncate1_T")
    T = T.permute([1, 0, 3, 2], rowrank=2)
    S, charges, U, vT = OS.svd_truncate(T, 200, 0.0)
    got = np.sort(np.concatenate(S))
    ans = np.sort(load_golden("svd_truncate1_S")["S"].reshape(-1))
    assert got.shape == ans.shape
    assert np.max(np.abs(got - ans)) < 1e-5


@pytest.mark.parametrize("minblock", [None, [1, 1, 0, 2, 0]])
def test_u1_exp_svals_truncation_matches_reference(minblock):
    T = golden_oracle_tensor("svd_u1_exp_src")
    suffix = "" if minblock is None else "_minblockdim"
    if minblock is None:
        S, charges, U, vT = OS.svd_truncate(T, 5, 0.0)
    else:
        S, charges, U, vT = OS.gesvd_truncate(T, 5, minblock, 0.0)
    q_ans, s_ans = _ans_sectors("svd_u1_exp_ans" + suffix)
    assert [c[0] for c in charges] == q_ans
    diff = np.sqrt(sum(float(np.sum((a - b) ** 2)) for a, b in zip(S, s_ans)))
    norm = max(1.0, np.sqrt(sum(float(np.sum(b ** 2)) for b in s_ans)))
    assert diff / norm < 1e-14
    assert U.labels == ["a", "b", "_aux_L"] and vT.labels == ["_aux_R", "c", "d"]
    rec = OS.recompose(U, S, vT, charges)
    ref = golden_oracle_tensor("svd_u1_exp_ans" + suffix + "_reconstructed")
    assert np.array_equal(rec.itoi, ref.itoi)
    d = rec.flat() - ref.flat()
    assert np.linalg.norm(d) <= 1e-14 * max(1.0, np.linalg.norm(ref.flat())) * 10
