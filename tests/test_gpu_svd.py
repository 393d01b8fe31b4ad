"""Block Svd_truncate / Gesvd_truncate on the device path against the reference's fixtures
and the oracle (oracle/svd.py, itself pinned to the same fixtures on the CPU):
Svd_truncate1 -> S_truncate1 (tests/linalg_test/linalg_test.cpp:57-67), the U(1)
exponentially-decaying case with keepdim 5 and with min_blockdim {1,1,0,2,0}
(tests/linalg_test/Gesvd_truncate_test.cpp:107-135), and the configuration-2 ground state
(D=1024) truncated back to D against the oracle."""
import numpy as np
import pytest
import torch

from conftest import golden_oracle_tensor, load_golden
from oracle import svd as OS

pytestmark = pytest.mark.gpu


def to_device(ot, c):
    bonds = [c.Bond(b.type, b.qnums, b.degs, [c.Symmetry(s[0], s[1]) for s in b.syms]) for b in ot.bonds]
    u = c.UniTensor(bonds, labels=ot.labels, rowrank=ot.rowrank, device=0)
    idx = u._layout.index()
    for t, blk in zip(ot.itoi.tolist(), ot.blocks):
        b = idx[tuple(t)]
        off = int(u._layout.offs[b])
        u._data[off: off + blk.size] = torch.from_numpy(np.ascontiguousarray(blk, dtype=np.float64).reshape(-1)).cuda()
    return u


def s_sectors(S):
    """(charges, per-sector singular values) of a square-diagonal-block S."""
    q = [int(x) for x in S.bonds()[0]._qnums[:, 0]]
    vals = []
    for b in range(S.Nblocks()):
        blk = S.get_block_(b).numpy()
        vals.append(np.diag(blk).copy())
    return q, vals


def test_svd_truncate1_reference_values():
    import cytnx_b200 as c

    T = to_device(golden_oracle_tensor("svd_truncate1_T"), c)
    T.permute_([1, 0, 3, 2])
    T.contiguous_()
    T.set_rowrank_(2)
    S, U, Vt = c.linalg.Svd_truncate(T, 200, 0.0, True)
    got = np.sort(np.concatenate(s_sectors(S)[1]))
    ans = np.sort(load_golden("svd_truncate1_S")["S"].reshape(-1))
    assert got.shape == ans.shape
    assert np.max(np.abs(got - ans)) < 1e-5
    # the fixture stores Float data; both sides compute on its FP64 conversion
    To = golden_oracle_tensor("svd_truncate1_T").astype(np.float64).permute([1, 0, 3, 2], rowrank=2)
    So, qo, _, _ = OS.svd_truncate(To, 200, 0.0)
    q, vals = s_sectors(S)
    assert q == [x[0] for x in qo]
    for a, b in zip(vals, So):
        assert np.allclose(a, b, rtol=0, atol=1e-12 * max(1.0, b.max()))


@pytest.mark.parametrize("minblock", [None, [1, 1, 0, 2, 0]])
def test_u1_exp_svals_reference_fixtures(minblock):
    import cytnx_b200 as c

    T = to_device(golden_oracle_tensor("svd_u1_exp_src"), c)
    suffix = "" if minblock is None else "_minblockdim"
    if minblock is None:
        S, U, Vt = c.linalg.Gesvd_truncate(T, 5, 0.0, True, True, 0)
    else:
        S, U, Vt = c.linalg.Gesvd_truncate(T, 5, minblock, 0.0, True, True, 0)
    z = load_golden("svd_u1_exp_ans" + suffix)
    q_ans = [int(x) for x in z["bond0_qnums"].reshape(-1)]
    pos, s_ans = 0, []
    for shp in z["block_shapes"]:
        n = int(np.prod(shp))
        s_ans.append(z["data"][pos:pos + n])
        pos += n
    q, vals = s_sectors(S)
    assert q == q_ans
    diff = np.sqrt(sum(float(np.sum((a - b) ** 2)) for a, b in zip(vals, s_ans)))
    assert diff / max(1.0, np.sqrt(sum(float(np.sum(b ** 2)) for b in s_ans))) < 1e-14
    assert U.labels() == ["a", "b", "_aux_L"] and Vt.labels() == ["_aux_R", "c", "d"]
    rec = c.Contract(c.Contract(U, S), Vt).permute(["a", "b", "c", "d"]).contiguous()
    ref = golden_oracle_tensor("svd_u1_exp_ans" + suffix + "_reconstructed")
    assert np.array_equal(rec._layout.itoi, ref.itoi)
    d = rec.flat_view().cpu().numpy() - ref.flat()
    assert np.linalg.norm(d) <= 1e-13 * max(1.0, np.linalg.norm(ref.flat()))


def test_config2_ground_state_truncation_matches_oracle():
    """Svd_truncate of a D=1024 two-site state (rowrank 2: (a, s1) | (s2, b)) back to D:
    the kept singular values of every sector equal the oracle's to 1e-12."""
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W
    import oracle as O
    from oracle import workloads as OW

    psi, L, M1, M2, R = W.build_two_site(W.xxz_spec(1024), W.xxz_mpo_values(), seed=0, device=0)
    psi.set_rowrank_(2)
    S, U, Vt = c.linalg.Svd_truncate(psi, 1024)
    ops = OW.xxz_two_site(1024, seed=0)
    p = ops["psi"]
    po = O.BlockTensor(p.bonds, p.labels, 2, p.itoi, p.blocks)
    So, qo, _, _ = OS.svd_truncate(po, 1024)
    q, vals = s_sectors(S)
    assert q == [x[0] for x in qo]
    for a, b in zip(vals, So):
        assert a.shape == b.shape
        assert np.max(np.abs(a - b)) <= 1e-12 * max(1.0, b.max())
