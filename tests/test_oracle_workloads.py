"""The oracle's own builder of the benchmark inputs (oracle/workloads.py, numpy + the
oracle's block enumeration) against the product's builder: identical block order and
identical values for the same seed, and the same algorithmic flop count.  The CPU
baseline and the bench's reference arm use the oracle builder only."""
import numpy as np
import pytest

import oracle as O
from oracle import workloads as OW


@pytest.mark.parametrize("D", [16, 64, 300])
def test_xxz_inputs_and_flops_match_product_builder(D):
    from cytnx_b200 import workloads as W
    from cytnx_b200.heff import _struct_contract
    from cytnx_b200.unitensor import contract_plan_flops

    spec = W.xxz_spec(D)
    psi, L, M1, M2, R = W.build_two_site(spec, W.xxz_mpo_values(), seed=3, device=-1)
    ops = OW.xxz_two_site(D, seed=3)
    for name, u in (("psi", psi), ("L", L), ("R", R), ("M1", M1), ("M2", M2)):
        assert np.array_equal(u._layout.itoi, ops[name].itoi), name
        assert np.array_equal(u._data.numpy(), ops[name].flat()), name
    # the product planner's flop count of the same four contractions
    t = L.relabels(["w", "a", "ap"])
    f = 0.0
    x = psi.relabels(["a", "s1", "s2", "b"])
    for a, b in ((t, x), (None, M1.relabels(["w", "w1", "s1", "s1p"])), (None, M2.relabels(["w1", "w2", "s2", "s2p"])),
                 (None, R.relabels(["w2", "b", "bp"]))):
        if a is None:
            a = cur
        f += contract_plan_flops(a, b)
        cur = _struct_contract(a, b)
    assert OW.heff_flops(ops) == f


def test_hubbard_inputs_match_product_builder():
    from cytnx_b200 import workloads as W

    dims = [40, 64, 200]
    for i, (p, D) in enumerate(zip(W.hubbard_batch(dims), dims)):
        l, r, x = W.problem_data(p, 1000 + i)
        ops = OW.hubbard_two_site(D, 1000 + i)
        Lc, _, _, Rc, Pc = p
        assert np.array_equal(Lc._layout.itoi, ops["L"].itoi)
        assert np.array_equal(Rc._layout.itoi, ops["R"].itoi)
        assert np.array_equal(Pc._layout.itoi, ops["psi"].itoi)
        assert np.array_equal(l.astype(np.float64), ops["L"].flat())
        assert np.array_equal(r.astype(np.float64), ops["R"].flat())
        assert np.array_equal(x.astype(np.float64), ops["psi"].flat())


def test_sampled_contractions_cover_the_matvec():
    """Pair sampling: the strided steps of one cycle multiply every block pair once."""
    ops = OW.xxz_two_site(64, seed=1)
    whole = OW.heff_flops(ops)
    outs = OW.heff_chain(ops)
    for stride in (1, 3, 7):
        fl = []
        for off in range(stride):
            OW.heff_chain(ops, stride=stride, offset=off, outs=outs, flops=fl)
        assert sum(fl) == whole


def test_oracle_matvec_is_the_network_contraction():
    """heff_matvec equals a dense contraction of the same network (small D)."""
    ops = OW.xxz_two_site(16, seed=2)
    y = OW.heff_matvec(ops)
    d = {k: v.dense() for k, v in ops.items()}
    ref = np.einsum("wap,asTb,wvsS,vuTU,ubq->pSUq", d["L"], d["psi"], d["M1"], d["M2"], d["R"], optimize=True)
    out = OW.with_psi(ops, y)["psi"].dense()
    assert np.linalg.norm(out - ref) <= 1e-12 * np.linalg.norm(ref)


def test_oracle_mps_heff_times_site_gives_the_energy():
    """<A_k, H_eff,k A_k> equals <psi|H|psi> of the dense state for every site k."""
    import itertools

    rng = np.random.default_rng(4)
    Ls = 5
    # bond k charges (sum of -2Sz over the left sites), total Sz = 0 on the last bond
    bond_q = [[0], [-1, 1], [-2, 0, 2], [-1, 1], [-2, 0, 2], [-1]]
    bond_d = [[1]] + [[2] * len(q) for q in bond_q[1:-1]] + [[1]]
    V = [O.Bond(-1, np.array(q).reshape(-1, 1), d) for q, d in zip(bond_q, bond_d)]
    phys = O.Bond(-1, np.array([1, -1]).reshape(-1, 1), [1, 1])
    flats, dense = [], []
    for j in range(Ls):
        bonds = [V[j], phys.redirect(), V[j + 1].redirect()]
        itoi = O.enumerate_blocks(bonds)
        n = sum(int(np.prod([bonds[i].degs[q] for i, q in enumerate(t)])) for t in itoi)
        f = rng.standard_normal(n)
        flats.append(f)
        dense.append(O.BlockTensor.from_flat(bonds, ["a", "s", "b"], 2, itoi, f).dense())
    psi = dense[0]
    for A in dense[1:]:
        psi = np.tensordot(psi, A, axes=([-1], [0]))
    psi = psi.reshape([2] * Ls)  # boundary bonds have dimension 1
    Wd = np.zeros((5, 5, 2, 2))
    for (w, wn, s, sp), v in OW.xxz_mpo_values().items():
        Wd[w, wn, s, sp] = v
    E = 0.0
    for s in itertools.product(range(2), repeat=Ls):
        for sp in itertools.product(range(2), repeat=Ls):
            vec = np.zeros(5)
            vec[0] = 1.0
            for i in range(Ls):
                vec = vec @ Wd[:, :, s[i], sp[i]]
            E += psi[s] * psi[sp] * vec[4]
    for k in range(Ls):
        y = OW.mps_heff_times_site(bond_q, bond_d, flats, k)
        assert abs(float(np.dot(flats[k], y)) - E) <= 1e-12 * max(1.0, abs(E))


def test_oracle_env_updates_are_the_networks():
    """env_left / env_right equal dense contractions of the example's networks (small D)."""
    ops = OW.xxz_two_site(16, seed=6)
    q, d = OW.u1_sector_sizes(16)
    A = OW.random_site(q, d, seed=2)
    Ld, Rd, Md, Ad = ops["L"].dense(), ops["R"].dense(), ops["M1"].dense(), A.dense()
    ref_l = np.einsum("wap,asb,wnsS,pSq->nbq", Ld, Ad, Md, Ad)
    got_l = OW.env_left(ops["L"], A, ops["M1"]).dense()
    assert np.linalg.norm(got_l - ref_l) <= 1e-12 * np.linalg.norm(ref_l)
    ref_r = np.einsum("asb,nbq,wnsS,pSq->wap", Ad, Rd, Md, Ad)
    got_r = OW.env_right(ops["R"], A, ops["M1"]).dense()
    assert np.linalg.norm(got_r - ref_r) <= 1e-12 * np.linalg.norm(ref_r)


def test_oracle_mps_energy_grad_matches_finite_differences():
    """The oracle's environment-sweep energy and gradient (config-5 CPU baseline) against
    central finite differences, and its H_eff A against mps_heff_times_site."""
    rng = np.random.default_rng(8)
    bond_q = [[0], [-1, 1], [-2, 0, 2], [-1, 1], [0]]
    bond_d = [[1], [2, 2], [1, 3, 1], [2, 2], [1]]
    flats = []
    for j in range(4):
        V0 = O.Bond(-1, np.array(bond_q[j]).reshape(-1, 1), bond_d[j])
        V1 = O.Bond(-1, np.array(bond_q[j + 1]).reshape(-1, 1), bond_d[j + 1])
        ph = O.Bond(-1, np.array([1, -1]).reshape(-1, 1), [1, 1])
        bonds = [V0, ph.redirect(), V1.redirect()]
        n = sum(int(np.prod([bonds[i].degs[q] for i, q in enumerate(t)])) for t in O.enumerate_blocks(bonds))
        flats.append(rng.standard_normal(n))
    num, den, grads = OW.mps_energy_grad(bond_q, bond_d, flats)
    for k in range(4):
        y = OW.mps_heff_times_site(bond_q, bond_d, flats, k)
        assert abs(float(np.dot(flats[k], y)) - num) <= 1e-12 * abs(num)
    h = 1e-6
    for k, i in ((0, 0), (2, 3), (3, 1)):
        fp = [f.copy() for f in flats]
        fm = [f.copy() for f in flats]
        fp[k][i] += h
        fm[k][i] -= h
        ep = OW.mps_energy_grad(bond_q, bond_d, fp)
        em = OW.mps_energy_grad(bond_q, bond_d, fm)
        fd = (ep[0] / ep[1] - em[0] / em[1]) / (2 * h)
        assert abs(fd - grads[k][i]) <= 1e-7 * max(1.0, abs(fd))
