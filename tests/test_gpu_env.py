"""Environment updates (cytnx_b200.env: left_update / right_update, the L A M A^dagger and
A R M A^dagger networks of example/DMRG/dmrg_two_sites_U1.py:115-126, 151-161) against the
oracle's contractions, at a U(1) bond dimension of 1024 (the configuration-2 sectors)."""
import numpy as np
import pytest
import torch

from oracle import workloads as OW

pytestmark = pytest.mark.gpu


def to_device(ot, c, labels=None):
    bonds = [c.Bond(b.type, b.qnums, b.degs, [c.Symmetry(s[0], s[1]) for s in b.syms]) for b in ot.bonds]
    u = c.UniTensor(bonds, labels=labels or ot.labels, rowrank=ot.rowrank, device=0)
    assert np.array_equal(u._layout.itoi, ot.itoi)
    u._data.copy_(torch.from_numpy(np.ascontiguousarray(ot.flat())).cuda())
    return u


def _check(got, ref):
    """Same blocks (matched by qnum tuple; the oracle keeps a permuted tensor's blocks in their
    old order, the product re-enumerates them) with the same values."""
    got = got.contiguous()
    assert sorted(map(tuple, got._layout.itoi.tolist())) == sorted(map(tuple, ref.itoi.tolist()))
    idx = {tuple(t): i for i, t in enumerate(ref.itoi.tolist())}
    g = np.concatenate([got.get_block_(b).numpy().ravel() for b in range(got.Nblocks())])
    r = np.concatenate([ref.blocks[idx[tuple(t)]].ravel() for t in got._layout.itoi.tolist()])
    assert np.linalg.norm(g - r) <= 1e-12 * np.linalg.norm(r)


@pytest.mark.parametrize("D", [64, 1024])
def test_left_and_right_updates_match_oracle(D):
    import cytnx_b200 as c
    from cytnx_b200 import env

    ops = OW.xxz_two_site(D, seed=3)
    q, d = OW.u1_sector_sizes(D)
    A = OW.random_site(q, d, seed=9)
    L = to_device(ops["L"], c, ["w", "a", "ap"])
    R = to_device(ops["R"], c, ["w", "b", "bp"])
    Ad = to_device(A, c)
    M = to_device(ops["M1"], c, ["w0", "w1", "s", "sp"])
    _check(env.left_update(L, Ad, M), OW.env_left(ops["L"], A, ops["M1"]))
    _check(env.right_update(R, Ad, M), OW.env_right(ops["R"], A, ops["M1"]))
    # chained: the result feeds the next update with the same structure
    L2 = env.left_update(env.left_update(L, Ad, M), Ad, M)
    _check(L2, OW.env_left(OW.env_left(ops["L"], A, ops["M1"]), A, ops["M1"]))
