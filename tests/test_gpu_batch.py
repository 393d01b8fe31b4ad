"""Batched two-site H_eff (many Hubbard problems, one launch per phase) against FP64.

Each problem's slice of the batched split-precision matvec is compared with the FP64
planned matvec of the same problem, which is itself checked against the oracle on a
Hubbard problem here; CUDA-graph replay must reproduce the eager launch bit for bit."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

DIMS = [40, 64, 96, 128, 200, 17, 256, 72]


def _problems(dims=DIMS, seed=11):
    from cytnx_b200 import workloads as W

    probs = W.hubbard_batch(dims)
    data = [W.problem_data(p, seed + i) for i, p in enumerate(probs)]
    return probs, data


def _fp64_reference(probs, data):
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    refs = []
    for (L, M1, M2, R, psi), (l, r, x) in zip(probs, data):
        Lg, Rg, Pg = W.materialize(L, l, 0), W.materialize(R, r, 0), W.materialize(psi, x, 0)
        H = c.TwoSiteHeff(Lg, M1, M2, Rg, Pg)  # MPO values are read on the host
        refs.append(H.matvec(Pg).flat_view().cpu().numpy())
    return refs


def _to_oracle(u, flat, labels):
    bonds = [O.Bond(b.type(), b._qnums, b._degs) for b in u.bonds()]
    lay = u._layout
    blocks = [np.asarray(flat[lay.offs[i]: lay.offs[i] + lay.sizes[i]], np.float64).reshape(lay.shapes[i])
              for i in range(len(lay.offs))]
    return O.BlockTensor(bonds, labels, u.rowrank(), lay.itoi, blocks)


def _slices(B, t):
    return torch.cat([t[int(o): int(o) + int(n)] for o, n in zip(B.psi_offsets, B.psi_sizes)])


def test_fp64_reference_matches_oracle_on_hubbard():
    probs, data = _problems([48], seed=5)
    (L, M, _, R, psi), (l, r, x) = probs[0], data[0]
    ref = _fp64_reference(probs, data)[0]
    m = M._data.cpu().numpy()
    ops = {"psi": _to_oracle(psi, x, ["-1", "-2", "-3", "-4"]), "L": _to_oracle(L, l, ["-5", "-1", "0"]),
           "R": _to_oracle(R, r, ["-7", "-4", "3"]), "M1": _to_oracle(M, m, ["-5", "-6", "-2", "1"]),
           "M2": _to_oracle(M, m, ["-6", "-7", "-3", "2"])}
    t = ops["L"].contract(ops["psi"])
    t = t.contract(ops["M1"]).contract(ops["M2"]).contract(ops["R"])
    t = t.permute([t.labels.index(k) for k in ["0", "1", "2", "3"]])
    assert np.array_equal(t.itoi, psi._layout.itoi)
    flat = np.concatenate([b.ravel() for b in t.blocks])
    assert np.linalg.norm(ref - flat) / np.linalg.norm(flat) < 1e-13


@pytest.mark.parametrize("precision", ["bf16x3", "3xtf32"])
@pytest.mark.parametrize("fp32", [True, False])
def test_batched_matvec_matches_fp64(precision, fp32):
    from cytnx_b200.batch import BatchedTwoSiteHeff

    probs, data = _problems()
    refs = _fp64_reference(probs, data)
    B = BatchedTwoSiteHeff(probs, precision, fp32=fp32)
    L_all = B.gather([d[0] for d in data], "L")
    R_all = B.gather([d[1] for d in data], "R")
    x_all = B.gather([d[2] for d in data], "psi")
    B.set_env(L_all, R_all)
    y = B.matvec(x_all, torch.zeros_like(x_all))
    torch.cuda.synchronize()
    yh = y.double().cpu().numpy()
    for i, ref in enumerate(refs):
        got = yh[B.psi_offsets[i]: B.psi_offsets[i] + B.psi_sizes[i]]
        err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
        # split products accumulated in FP32: ~1e-6 relative (BF16x3 of FP32 data: ~7e-6)
        assert err < 2e-5, (i, DIMS[i], err)
    # elements between the problems' slices are left as they were (zero)
    mask = np.ones(B.psi_total, bool)
    for i in range(B.nprob):
        mask[B.psi_offsets[i]: B.psi_offsets[i] + B.psi_sizes[i]] = False
    assert not np.any(yh[mask])


def test_graph_replay_is_bitwise_and_tracks_inputs():
    from cytnx_b200.batch import BatchedTwoSiteHeff

    probs, data = _problems()
    B = BatchedTwoSiteHeff(probs, "bf16x3")
    B.set_env(B.gather([d[0] for d in data], "L"), B.gather([d[1] for d in data], "R"))
    x_all = B.gather([d[2] for d in data], "psi")
    out = torch.zeros_like(x_all)
    B.capture(x_all, out)
    eager = B.matvec(x_all.clone(), torch.zeros_like(x_all))
    out.fill_(7.0)
    B.replay()
    torch.cuda.synchronize()
    assert torch.equal(_slices(B, out), _slices(B, eager))
    # new contents of the captured input buffer flow through the replay
    x_all.mul_(-2.0)
    B.replay()
    eager2 = B.matvec(x_all.clone(), torch.zeros_like(x_all))
    torch.cuda.synchronize()
    assert torch.equal(_slices(B, out), _slices(B, eager2))
    assert torch.equal(_slices(B, out), -2.0 * _slices(B, eager))


def test_autotune_keeps_results():
    from cytnx_b200.batch import BatchedTwoSiteHeff

    probs, data = _problems(DIMS[:5])
    refs = _fp64_reference(probs, data)
    B = BatchedTwoSiteHeff(probs, "3xtf32")
    B.set_env(B.gather([d[0] for d in data], "L"), B.gather([d[1] for d in data], "R"))
    x_all = B.gather([d[2] for d in data], "psi")
    res = B.autotune(x_all, step1=(96, 128), step4=(32, 48, 64), reps=2)
    assert res["step1"] in (96, 128) and res["step4"] in (32, 48, 64)
    assert B.tiles == (res["step1"], res["step4"])
    y = B.matvec(x_all).double().cpu().numpy()
    for i, ref in enumerate(refs):
        got = y[B.psi_offsets[i]: B.psi_offsets[i] + B.psi_sizes[i]]
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 2e-5


def test_batched_problems_match_oracle():
    """Eight Hubbard problems of different D (17 .. 256): the FP64 planned matvec to
    1e-12 and every split form's slice of the batched launch against the oracle's FP64
    matvec of the same FP32-valued inputs (built by the oracle's own generator)."""
    from cytnx_b200.batch import BatchedTwoSiteHeff
    from oracle import workloads as OW

    probs, data = _problems()
    refs = [OW.heff_matvec(OW.hubbard_two_site(D, 11 + i)) for i, D in enumerate(DIMS)]
    for got, ref in zip(_fp64_reference(probs, data), refs):
        assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12
    for precision, bound in (("bf16x3", 2e-5), ("3xtf32", 3e-6)):
        B = BatchedTwoSiteHeff(probs, precision, fp32=True)
        B.set_env(B.gather([d[0] for d in data], "L"), B.gather([d[1] for d in data], "R"))
        x_all = B.gather([d[2] for d in data], "psi")
        y = B.matvec(x_all, torch.zeros_like(x_all)).double().cpu().numpy()
        for i, ref in enumerate(refs):
            got = y[B.psi_offsets[i]: B.psi_offsets[i] + B.psi_sizes[i]]
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err <= bound, (precision, DIMS[i], err)
