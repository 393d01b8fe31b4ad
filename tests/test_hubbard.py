"""Host-side checks of the batched Hubbard workload: the MPO against an exact Fock-space
Hamiltonian, the (N, 2Sz) sector generator, and batch planning (no GPU needed)."""
import itertools

import numpy as np
import pytest
import torch

from cytnx_b200 import workloads as W


def _mpo_dense(nsites, vals, nw=6):
    Mt = np.zeros((nw, nw, 4, 4))
    for (a, b, s, sp), v in vals.items():
        Mt[a, b, s, sp] = v
    dim = 4 ** nsites
    H = np.zeros((dim, dim))
    for sin in itertools.product(range(4), repeat=nsites):
        for sout in itertools.product(range(4), repeat=nsites):
            v = np.zeros(nw)
            v[0] = 1.0
            for i in range(nsites):
                v = v @ Mt[:, :, sin[i], sout[i]]
            ii = sum(s * 4 ** (nsites - 1 - i) for i, s in enumerate(sin))
            oo = sum(s * 4 ** (nsites - 1 - i) for i, s in enumerate(sout))
            H[oo, ii] = v[nw - 1]
    return H


def _fock_hubbard(nsites, U, t):
    """H from fermion operators on 2*nsites modes ordered (1up, 1dn, 2up, ...), built by
    enumerating occupations with the anticommutation sign of each annihilator."""
    dim = 4 ** nsites

    def occ(sites):
        o = []
        for s in sites:  # site state s = n_up + 2 n_dn
            o += [s & 1, (s >> 1) & 1]
        return o

    def index(o):
        return sum((o[2 * i] + 2 * o[2 * i + 1]) * 4 ** (nsites - 1 - i) for i in range(nsites))

    def annihilator(k):
        C = np.zeros((dim, dim))
        for sites in itertools.product(range(4), repeat=nsites):
            o = occ(sites)
            if o[k]:
                o2 = list(o)
                o2[k] = 0
                C[index(o2), index(o)] = (-1) ** sum(o[:k])
        return C

    c = [annihilator(k) for k in range(2 * nsites)]
    H = np.zeros((dim, dim))
    for i in range(nsites - 1):
        for sg in range(2):
            a, b = c[2 * i + sg], c[2 * (i + 1) + sg]
            H += -t * (a.T @ b + b.T @ a)
    for i in range(nsites):
        H += U * (c[2 * i].T @ c[2 * i]) @ (c[2 * i + 1].T @ c[2 * i + 1])
    return H


@pytest.mark.parametrize("U,t", [(4.0, 1.0), (2.5, -0.7)])
def test_hubbard_mpo_matches_fock_space(U, t):
    H_mpo = _mpo_dense(3, W.hubbard_mpo_values(U, t))
    H_ref = _fock_hubbard(3, U, t)
    assert np.array_equal(H_mpo, H_ref)


def test_hubbard_two_site_half_filling_energy():
    """Two-site Hubbard dimer at N=2: E0 = (U - sqrt(U^2 + 16 t^2)) / 2."""
    H = _mpo_dense(2, W.hubbard_mpo_values(4.0, 1.0))
    nsec = [sum(W.HUB_PHYS_Q[s][0] for s in (i // 4, i % 4)) for i in range(16)]
    idx = [i for i in range(16) if nsec[i] == 2]
    e0 = np.linalg.eigvalsh(H[np.ix_(idx, idx)])[0]
    assert abs(e0 - (4.0 - np.sqrt(32.0)) / 2) < 1e-12


def test_hubbard_mpo_respects_charges():
    phys, inner = np.array(W.HUB_PHYS_Q), np.array(W.HUB_INNER_Q)
    for (w0, w1, s, sp) in W.hubbard_mpo_values():
        # M[w_in ket, w_out bra, s ket, s' bra]: q(w_in) + q(s) - q(w_out) - q(s') = 0
        assert np.array_equal(inner[w0] + phys[s] - inner[w1] - phys[sp], [0, 0])


@pytest.mark.parametrize("D", [128, 777, 2048])
def test_hubbard_sectors(D):
    q, d = W.hubbard_sector_sizes(D)
    assert d.sum() == D and (d > 0).all()
    assert ((q[:, 0] - q[:, 1]) % 2 == 0).all()
    assert len({tuple(x) for x in q.tolist()}) == len(q)
    sizes = {tuple(x): int(n) for x, n in zip(q.tolist(), d)}
    assert sizes[(0, 0)] == max(sizes.values())


def test_batch_dims_seeded():
    a, b = W.hubbard_batch_dims(256, seed=0), W.hubbard_batch_dims(256, seed=0)
    assert a == b and min(a) >= 128 and max(a) <= 2048 and len(a) == 256


@pytest.mark.parametrize("prec", ["bf16x3", "3xtf32"])
def test_batch_planning_host_only(prec):
    """Planning and batch table concatenation are host work: flops add up over problems."""
    from cytnx_b200 import _lib
    from cytnx_b200.batch import BatchedTwoSiteHeff

    dims = [24, 40, 64, 33]
    probs = W.hubbard_batch(dims)
    B = BatchedTwoSiteHeff(probs, prec, device=torch.device("cpu"))
    assert B.nprob == 4
    assert (B.psi_offsets % 32 == 0).all() and (B.L_offsets % 32 == 0).all()
    tot = 0.0
    for i in range(4):
        h = B.plan(i)
        tot += _lib.lib().ctn_heff2_split_gemm_flops(h, B.prec, 1) + _lib.lib().ctn_heff2_split_gemm_flops(h, B.prec, 4)
    assert tot > 0 and abs(B.gemm_flops() - tot) <= 1e-9 * tot
    assert B.workspace_bytes() > 0
    for i, (L, _, _, R, psi) in enumerate(probs):
        assert B.psi_sizes[i] == psi._layout.nelem
        assert B.L_sizes[i] == L._layout.nelem and B.R_sizes[i] == R._layout.nelem
    # tile widths are validated before any table is built
    with pytest.raises(Exception):
        B._create(100, 64)


def test_mps_bond_sectors():
    from cytnx_b200.autodiff import mps_bond_sectors

    for L, Dmax in ((32, 512), (10, 16), (8, 1000)):
        for k in range(L + 1):
            q, d = mps_bond_sectors(L, k, Dmax)
            assert d.sum() <= Dmax and (d > 0).all()
            assert ((q + k) % 2 == 0).all() and (np.abs(q) <= min(k, L - k)).all()
        q0, d0 = mps_bond_sectors(L, 0, Dmax)
        qL, dL = mps_bond_sectors(L, L, Dmax)
        assert q0.tolist() == [0] and d0.tolist() == [1] and qL.tolist() == [0] and dL.tolist() == [1]
    # no cap binds: exact Schmidt dimensions
    q, d = mps_bond_sectors(8, 4, 1000)
    assert dict(zip(q.tolist(), d.tolist())) == {-4: 1, -2: 4, 0: 6, 2: 4, 4: 1}


def test_redirected_bonds_keep_the_block_layout():
    from cytnx_b200.unitensor import layout_for

    spec = W.xxz_spec(64)
    Vl, Vr, phys, inner = W.spec_bonds(spec)
    bonds = [inner.redirect(), Vl.redirect(), Vl]
    a, b = layout_for(bonds), layout_for([x.redirect() for x in bonds])
    assert np.array_equal(a.itoi, b.itoi) and np.array_equal(a.offs, b.offs)
