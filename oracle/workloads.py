"""Seeded synthetic inputs of the benchmark configurations, built for the oracle --
TEST INFRASTRUCTURE, never part of the product.

The reference has no generator for these problems (its DMRG example starts from random
tensors of its own RNG, ``example/DMRG/dmrg_two_sites_U1.py``), so this module states
the synthetic-input rules once more, independently of the product package: numpy
(PCG64, seeded) for the values and the oracle's own block enumeration
(``BlockUniTensor.cpp:190-230`` restated in ``oracle.c``) for the block order.  Given
the same seed it yields bit for bit the values the product's workload builder places
on the device (a CPU test checks that), so the oracle and the CUDA path see identical
inputs while the CPU baseline imports nothing from the product.

* ``u1_sector_sizes``    sector sizes ~ exp(-q^2/72), q = -16..16, largest remainder to D.
* ``xxz_mpo_values``     the spin-1/2 XXZ MPO (bond dimension 5) in the leg convention of
                         ``example/DMRG/dmrg_two_sites_U1.py:43-60``.
* ``xxz_two_site``       L[w,a,a'], R[w,b,b'] (Hermitian), psi[a,s1,s2,b] (normalised), M1, M2.
* ``hubbard_*``          the batched Hubbard problems (U=4, t=1, d=4, (N, 2Sz) charges).
* ``heff_matvec``        the two-site H_eff matvec of ``dmrg_two_sites_U1.py:18-34`` as four
                         pairwise ``BlockTensor.contract`` calls in the order L -> M1 -> M2 -> R
                         (the network's ORDER-free left fold starting from psi and L).
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import Bond, BlockTensor, enumerate_blocks

NET = {"psi": ["-1", "-2", "-3", "-4"], "L": ["-5", "-1", "0"], "R": ["-7", "-4", "3"],
       "M1": ["-5", "-6", "-2", "1"], "M2": ["-6", "-7", "-3", "2"]}
TOUT = ["0", "1", "2", "3"]

KET, BRA = -1, 1


def u1_sector_sizes(D: int, qmax: int = 16, var: float = 72.0):
    q = np.arange(-qmax, qmax + 1)
    w = np.exp(-(q.astype(np.float64) ** 2) / var)
    raw = D * w / w.sum()
    base = np.floor(raw).astype(np.int64)
    rem = D - int(base.sum())
    order = sorted(range(len(q)), key=lambda i: (-(raw[i] - base[i]), abs(q[i]), q[i]))
    for i in order[:rem]:
        base[i] += 1
    keep = base > 0
    return q[keep].astype(np.int64), base[keep]


def xxz_mpo_values(Jz: float = 1.0, Jxy: float = 1.0, h: float = 0.0) -> Dict[Tuple[int, int, int, int], float]:
    """Nonzero M[w_in, w_out, s, s'] = coefficient * <s'|O|s>; s = 0 up (+1), 1 down (-1)."""
    c = np.sqrt(abs(Jxy) / 2.0)
    sgn = 1.0 if Jxy >= 0 else -1.0
    m = {}
    for s, sz in ((0, 0.5), (1, -0.5)):
        m[(0, 0, s, s)] = 1.0
        m[(4, 4, s, s)] = 1.0
        m[(0, 3, s, s)] = sz
        m[(3, 4, s, s)] = Jz * sz
        if h:
            m[(0, 4, s, s)] = h * sz
    m[(0, 1, 1, 0)] = c
    m[(1, 4, 0, 1)] = sgn * c
    m[(0, 2, 0, 1)] = c
    m[(2, 4, 1, 0)] = sgn * c
    return m


XXZ_INNER_Q = [0, -2, 2, 0, 0]
XXZ_P = [0, 2, 1, 3, 4]
SPIN_PHYS_Q = [1, -1]


def _col(q):
    a = np.asarray(q, dtype=np.int64)
    return a.reshape(-1, 1) if a.ndim == 1 else a


def _mpo(inner: Bond, phys: Bond, values, labels) -> BlockTensor:
    bonds = [inner, inner.redirect(), phys, phys.redirect()]
    itoi = enumerate_blocks(bonds)
    index = {tuple(t): i for i, t in enumerate(itoi.tolist())}
    flat = np.zeros(len(itoi))  # every block is 1 x 1 x 1 x 1
    for key, val in values.items():
        b = index.get(key)
        if b is None:
            raise ValueError(f"MPO entry {key} violates the symmetry")
        flat[b] = val
    return BlockTensor.from_flat(bonds, labels, 2, itoi, flat)


def two_site(qv, dv, qv_r, dv_r, phys_q, inner_q, P, mpo_values, seed: int, hermitian: bool = True,
             env_psi=None) -> Dict[str, BlockTensor]:
    """(psi, L, M1, M2, R) as oracle BlockTensors with the network labels of ``NET``.

    Value order (PCG64 from ``seed``): L's flat data, R's flat data, psi's flat data,
    each in block-enumeration order; L and R are then made Hermitian
    (L[w,a,a'] <- (L[w,a,a'] + L[P w,a',a]) / 2), psi is normalised.  ``env_psi`` instead
    gives the flat (L, R, psi) data (the batched problems draw their own)."""
    nsym = _col(qv).shape[1]
    syms = [(-1, 1)] * nsym
    Vl = Bond(KET, _col(qv), dv, syms)
    Vr = Bond(KET, _col(qv_r), dv_r, syms)
    phys = Bond(KET, _col(phys_q), [1] * len(phys_q), syms)
    inner = Bond(KET, _col(inner_q), [1] * len(inner_q), syms)
    b_psi = [Vl, phys.redirect(), phys.redirect(), Vr.redirect()]
    b_L = [inner.redirect(), Vl.redirect(), Vl]
    b_R = [inner, Vr, Vr.redirect()]
    it_psi, it_L, it_R = enumerate_blocks(b_psi), enumerate_blocks(b_L), enumerate_blocks(b_R)

    def nelem(bonds, itoi):
        return int(sum(np.prod([bonds[i].degs[q] for i, q in enumerate(t)]) for t in itoi))

    if env_psi is None:
        rng = np.random.default_rng(seed)
        l = rng.standard_normal(nelem(b_L, it_L))
        r = rng.standard_normal(nelem(b_R, it_R))
        x = rng.standard_normal(nelem(b_psi, it_psi))
        x /= np.linalg.norm(x)
    else:
        l, r, x = (np.asarray(v, dtype=np.float64) for v in env_psi)
    L = BlockTensor.from_flat(b_L, NET["L"], 1, it_L, l)
    R = BlockTensor.from_flat(b_R, NET["R"], 1, it_R, r)
    if hermitian and env_psi is None:
        for T in (L, R):
            idx = {tuple(t): i for i, t in enumerate(T.itoi.tolist())}
            src = [b.copy() for b in T.blocks]
            for i, (w, a, b) in enumerate(T.itoi.tolist()):
                T.blocks[i][...] = 0.5 * (src[i] + src[idx[(P[w], b, a)]].transpose(0, 2, 1))
    psi = BlockTensor.from_flat(b_psi, NET["psi"], 1, it_psi, x)
    M1 = _mpo(inner, phys, mpo_values, NET["M1"])
    M2 = _mpo(inner, phys, mpo_values, NET["M2"])
    return {"psi": psi, "L": L, "R": R, "M1": M1, "M2": M2}


def xxz_two_site(D: int, seed: int = 0, Jz: float = 1.0, Jxy: float = 1.0, h: float = 0.0):
    """The U(1) XXZ two-site problem at bond dimension D (configurations 2 and 3)."""
    qv, dv = u1_sector_sizes(D)
    return two_site(qv, dv, qv, dv, SPIN_PHYS_Q, XXZ_INNER_Q, XXZ_P, xxz_mpo_values(Jz, Jxy, h), seed)


def with_psi(ops: Dict[str, BlockTensor], flat) -> Dict[str, BlockTensor]:
    """The same operators with psi's values replaced by ``flat``."""
    p = ops["psi"]
    return dict(ops, psi=BlockTensor.from_flat(p.bonds, p.labels, p.rowrank, p.itoi, np.asarray(flat, np.float64)))


def heff_chain(ops: Dict[str, BlockTensor], stride: int = 1, offset: int = 0, outs=None, flops=None):
    """The four pairwise contractions L.psi, .M1, .M2, .R (each result feeds the next).
    Returns the intermediates [T1, T2, T3, T4]; ``stride``/``offset``/``outs`` sample the
    block pairs of every step (``BlockTensor.contract``)."""
    res, t = [], ops["psi"]
    for k, name in enumerate(("L", "M1", "M2", "R")):
        o = outs[k] if outs is not None else None
        if name == "L":
            t = ops["L"].contract(t, stride=stride, offset=offset, out=o, flops=flops)
        else:
            t = t.contract(ops[name], stride=stride, offset=offset, out=o, flops=flops)
        res.append(t)
    return res


def heff_matvec(ops: Dict[str, BlockTensor], flat=None) -> np.ndarray:
    """H_eff psi (flat, in psi's block order) for psi = ``flat`` (default: ops' psi)."""
    o = ops if flat is None else with_psi(ops, flat)
    t = heff_chain(o)[-1]
    t = t.permute([t.labels.index(k) for k in TOUT])
    if not np.array_equal(t.itoi, o["psi"].itoi):
        raise RuntimeError("H_eff output blocks are not in psi's order")
    return t.flat()


def heff_flops(ops: Dict[str, BlockTensor]) -> float:
    """Algorithmic flops of one matvec: 2*M*N*K over every block pair of the four steps."""
    f = []
    t = ops["psi"]
    for name in ("L", "M1", "M2", "R"):
        if name == "L":
            f.append(ops["L"].contract_flops(t))
            t = ops["L"].contract(t, stride=0)
        else:
            f.append(t.contract_flops(ops[name]))
            t = t.contract(ops[name], stride=0)
    return float(sum(f))


# ---------------------------------------------------------------- spinful Hubbard chain
HUB_PHYS_Q = [(0, 0), (1, 1), (1, -1), (2, 0)]
HUB_INNER_Q = [(0, 0), (-1, -1), (-1, 1), (1, 1), (1, -1), (0, 0)]
HUB_P = [0, 3, 4, 1, 2, 5]


def hubbard_mpo_values(U: float = 4.0, t: float = 1.0, mu: float = 0.0):
    """M[w_in, w_out, s, s'] of H = -t sum (c+_i c_{i+1} + h.c.) + U sum n_up n_dn - mu sum n
    with Jordan-Wigner strings; basis |0>, |up>, |dn>, |updn> = c+_up c+_dn |0>."""
    cu = np.zeros((4, 4))
    cu[0, 1] = 1.0
    cu[2, 3] = 1.0
    cd = np.zeros((4, 4))
    cd[0, 2] = 1.0
    cd[1, 3] = -1.0
    F = np.diag([1.0, -1.0, -1.0, 1.0])
    nu, nd, I = cu.T @ cu, cd.T @ cd, np.eye(4)
    ops = {(0, 0): I, (5, 5): I, (0, 1): cu.T @ F, (1, 5): -t * cu, (0, 2): cd.T @ F, (2, 5): -t * cd,
           (0, 3): cu @ F, (3, 5): t * cu.T, (0, 4): cd @ F, (4, 5): t * cd.T,
           (0, 5): U * (nu @ nd) - mu * (nu + nd)}
    m = {}
    for (w0, w1), O in ops.items():
        for s in range(4):
            for sp in range(4):
                if O[sp, s] != 0.0:
                    m[(w0, w1, s, sp)] = float(O[sp, s])
    return m


def hubbard_sector_sizes(D: int, sigma: float = 4.0, center=(0, 0)):
    r = int(np.ceil(4 * sigma))
    pts = [(n, m) for n in range(-r, r + 1) for m in range(-r, r + 1) if (n - m) % 2 == 0]
    w = np.array([np.exp(-(n * n + m * m) / (2.0 * sigma * sigma)) for n, m in pts])
    raw = D * w / w.sum()
    base = np.floor(raw).astype(np.int64)
    rem = D - int(base.sum())
    order = sorted(range(len(pts)), key=lambda i: (-(raw[i] - base[i]), abs(pts[i][0]) + abs(pts[i][1]), pts[i]))
    for i in order[:rem]:
        base[i] += 1
    keep = base > 0
    q = np.array([(n + center[0], m + center[1]) for n, m in pts], dtype=np.int64)[keep]
    return q, base[keep]


def hubbard_batch_dims(nprob: int = 256, dmin: int = 128, dmax: int = 2048, seed: int = 0) -> List[int]:
    rng = np.random.default_rng(seed)
    return [int(d) for d in rng.integers(dmin, dmax + 1, size=nprob)]


def hubbard_two_site(D: int, seed: int, U: float = 4.0, t: float = 1.0, sigma: float = 4.0):
    """One batched Hubbard problem: left bond around (0, 0), right bond around (-2, 0);
    L, R, psi ~ N(0,1) rounded to FP32 values (psi normalised first), drawn L, R, psi."""
    ql, dl = hubbard_sector_sizes(D, sigma, (0, 0))
    qr, dr = hubbard_sector_sizes(D, sigma, (-2, 0))
    nl, nr, nx = (_nel(ql, dl, qr, dr, w) for w in ("L", "R", "psi"))
    rng = np.random.default_rng(seed)
    l = rng.standard_normal(nl).astype(np.float32)
    r = rng.standard_normal(nr).astype(np.float32)
    x = rng.standard_normal(nx)
    x = (x / np.linalg.norm(x)).astype(np.float32)
    return two_site(ql, dl, qr, dr, HUB_PHYS_Q, HUB_INNER_Q, HUB_P, hubbard_mpo_values(U, t), 0,
                    env_psi=(l, r, x))


def _nel(ql, dl, qr, dr, which):
    syms = [(-1, 1)] * 2
    Vl, Vr = Bond(KET, ql, dl, syms), Bond(KET, qr, dr, syms)
    phys = Bond(KET, _col(HUB_PHYS_Q), [1] * 4, syms)
    inner = Bond(KET, _col(HUB_INNER_Q), [1] * 6, syms)
    bonds = {"psi": [Vl, phys.redirect(), phys.redirect(), Vr.redirect()], "L": [inner.redirect(), Vl.redirect(), Vl],
             "R": [inner, Vr, Vr.redirect()]}[which]
    itoi = enumerate_blocks(bonds)
    return int(sum(np.prod([bonds[i].degs[q] for i, q in enumerate(t)]) for t in itoi))


# ---------------------------------------------------------------- finite U(1) MPS (differentiation check)
def mps_heff_times_site(bond_q, bond_d, site_flats, k: int, mpo_values=None, phys_q=SPIN_PHYS_Q,
                        inner_q=XXZ_INNER_Q, left_channel: int = 0, right_channel: int = 4) -> np.ndarray:
    """H_eff,k A_k for a finite MPS A_j[a (ket), s (bra), b (bra)] (flat data in block order)
    with the environments built by pairwise contractions, as the DMRG example builds them
    (``example/DMRG/dmrg_two_sites_U1.py:115-126`` for the left sweep, ``:151-161`` for the
    right):  L_{j+1} = ((L_j A_j) M) A_j^dagger,  R_{j-1} = ((A_j R_j) M) A_j^dagger,
    H_eff,k A_k = ((L_k A_k) M) R_k.  Real data: A^dagger carries A's values on the
    redirected bonds.  Returns the result flat in A_k's block order (legs a, s, b)."""
    mpo_values = xxz_mpo_values() if mpo_values is None else mpo_values
    Ls = len(site_flats)
    syms = [(-1, 1)]
    V = [Bond(KET, _col(q), d, syms) for q, d in zip(bond_q, bond_d)]
    phys = Bond(KET, _col(phys_q), [1] * len(phys_q), syms)
    inner = Bond(KET, _col(inner_q), [1] * len(inner_q), syms)
    M = _mpo(inner, phys, mpo_values, ["w", "wn", "s", "sp"])

    def site(j, labels, dagger=False):
        bonds = [V[j], phys.redirect(), V[j + 1].redirect()]
        itoi = enumerate_blocks(bonds)
        if dagger:
            bonds = [b.redirect() for b in bonds]
        return BlockTensor.from_flat(bonds, labels, 2, itoi, np.asarray(site_flats[j], np.float64))

    def unit(bonds, labels, tup):
        itoi = enumerate_blocks(bonds)
        flat = np.zeros(sum(int(np.prod([bonds[i].degs[q] for i, q in enumerate(t)])) for t in itoi))
        pos = [i for i, t in enumerate(itoi.tolist()) if tuple(t) == tuple(tup)]
        if len(pos) != 1:
            raise ValueError("boundary block not found")
        off = sum(int(np.prod([bonds[i].degs[q] for i, q in enumerate(t)])) for t in itoi[:pos[0]])
        flat[off] = 1.0
        return BlockTensor.from_flat(bonds, labels, 1, itoi, flat)

    Lenv = unit([inner.redirect(), V[0].redirect(), V[0]], ["w", "a", "ap"], (left_channel, 0, 0))
    for j in range(k):
        t = Lenv.contract(site(j, ["a", "s", "b"])).contract(M).contract(site(j, ["ap", "sp", "bp"], True))
        Lenv = t.relabel([{"b": "a", "wn": "w", "bp": "ap"}[l] for l in t.labels])
    Renv = unit([inner, V[Ls], V[Ls].redirect()], ["wn", "b", "bp"], (right_channel, 0, 0))
    for j in range(Ls - 1, k, -1):
        t = site(j, ["a", "s", "b"]).contract(Renv).contract(M).contract(site(j, ["ap", "sp", "bp"], True))
        Renv = t.relabel([{"w": "wn", "a": "b", "ap": "bp"}[l] for l in t.labels])
    Y = Lenv.contract(site(k, ["a", "s", "b"])).contract(M).contract(Renv)
    Y = Y.permute([Y.labels.index(l) for l in ("ap", "sp", "bp")])
    ref = site(k, ["a", "s", "b"])
    if not np.array_equal(Y.itoi, ref.itoi):
        raise RuntimeError("H_eff A_k blocks are not in A_k's order")
    return Y.flat()


def env_left(L: BlockTensor, A: BlockTensor, M: BlockTensor) -> BlockTensor:
    """L'[w, a, ap] = sum L[w,a,ap] A[a,s,b] M[w,wn,s,sp] A*[ap,sp,bp] (real data; legs by
    position), the left update of example/DMRG/dmrg_two_sites_U1.py:115-126, as the three
    pairwise contractions env . A, . M, . A^dagger.  Result legs (b -> a, wn -> w, bp -> ap) in the
    order [w, a, ap]."""
    Lr = L.relabel(["w", "a", "ap"])
    Ar = A.relabel(["a", "s", "b"])
    Ad = BlockTensor([b.redirect() for b in A.bonds], ["ap", "sp", "bp"], A.rowrank, A.itoi, A.blocks)
    t = Lr.contract(Ar).contract(M.relabel(["w", "wn", "s", "sp"])).contract(Ad)
    t = t.relabel([{"b": "a", "wn": "w", "bp": "ap"}[l] for l in t.labels])
    return t.permute([t.labels.index(l) for l in ("w", "a", "ap")])


def env_right(R: BlockTensor, A: BlockTensor, M: BlockTensor) -> BlockTensor:
    """R'[w, a, ap] = sum A[a,s,b] R[wn,b,bp] M[w,wn,s,sp] A*[ap,sp,bp] (real data; legs by
    position), the right update of example/DMRG/dmrg_two_sites_U1.py:151-161."""
    Rr = R.relabel(["wn", "b", "bp"])
    Ar = A.relabel(["a", "s", "b"])
    Ad = BlockTensor([b.redirect() for b in A.bonds], ["ap", "sp", "bp"], A.rowrank, A.itoi, A.blocks)
    t = Ar.contract(Rr).contract(M.relabel(["w", "wn", "s", "sp"])).contract(Ad)
    return t.permute([t.labels.index(l) for l in ("w", "a", "ap")])


def random_site(qv, dv, seed: int) -> BlockTensor:
    """A U(1) site tensor A[a (ket), s (bra), b (bra)] on the bond qv/dv at both ends, ~N(0,1)."""
    syms = [(-1, 1)]
    V = Bond(KET, _col(qv), dv, syms)
    phys = Bond(KET, _col(SPIN_PHYS_Q), [1, 1], syms)
    bonds = [V, phys.redirect(), V.redirect()]
    itoi = enumerate_blocks(bonds)
    n = sum(int(np.prod([bonds[i].degs[q] for i, q in enumerate(t)])) for t in itoi)
    return BlockTensor.from_flat(bonds, ["a", "s", "b"], 2, itoi, np.random.default_rng(seed).standard_normal(n))


def mps_energy_grad(bond_q, bond_d, site_flats, mpo_values=None, phys_q=SPIN_PHYS_Q, inner_q=XXZ_INNER_Q,
                    left_channel: int = 0, right_channel: int = 4):
    """<A|H|A>, <A|A> and the gradient of E = <A|H|A>/<A|A> for every site of a finite MPS
    (real data), by left and right environment sweeps of pairwise contractions (the
    example's networks): d<A|H|A>/dA_k = 2 H_eff,k A_k, d<A|A>/dA_k = 2 N_eff,k A_k, and
    dE/dA_k = (2 H_eff,k A_k - 2 E N_eff,k A_k) / <A|A>.  Returns (num, den, [grad_k flat])."""
    mpo_values = xxz_mpo_values() if mpo_values is None else mpo_values
    Ls = len(site_flats)
    syms = [(-1, 1)]
    V = [Bond(KET, _col(q), d, syms) for q, d in zip(bond_q, bond_d)]
    phys = Bond(KET, _col(phys_q), [1] * len(phys_q), syms)
    inner = Bond(KET, _col(inner_q), [1] * len(inner_q), syms)
    M = _mpo(inner, phys, mpo_values, ["w", "wn", "s", "sp"])

    def site(j, labels, dagger=False):
        bonds = [V[j], phys.redirect(), V[j + 1].redirect()]
        itoi = enumerate_blocks(bonds)
        if dagger:
            bonds = [b.redirect() for b in bonds]
        return BlockTensor.from_flat(bonds, labels, 2, itoi, np.asarray(site_flats[j], np.float64))

    def unit(bonds, labels, tup):
        itoi = enumerate_blocks(bonds)
        sizes = [int(np.prod([bonds[i].degs[q] for i, q in enumerate(t)])) for t in itoi]
        flat = np.zeros(sum(sizes))
        b = [i for i, t in enumerate(itoi.tolist()) if tuple(t) == tuple(tup)][0]
        flat[sum(sizes[:b])] = 1.0
        return BlockTensor.from_flat(bonds, labels, 1, itoi, flat)

    def relab(t, m):
        return t.relabel([m[l] for l in t.labels])

    HL = [unit([inner.redirect(), V[0].redirect(), V[0]], ["w", "a", "ap"], (left_channel, 0, 0))]
    NL = [unit([V[0].redirect(), V[0]], ["a", "ap"], (0, 0))]
    for j in range(Ls - 1):
        A, Ad = site(j, ["a", "s", "b"]), site(j, ["ap", "s", "bp"], True)
        t = HL[-1].contract(A).contract(M).contract(site(j, ["ap", "sp", "bp"], True))
        HL.append(relab(t, {"b": "a", "wn": "w", "bp": "ap"}))
        NL.append(relab(NL[-1].contract(A).contract(Ad), {"b": "a", "bp": "ap"}))
    HR = [None] * Ls
    NR = [None] * Ls
    HR[Ls - 1] = unit([inner, V[Ls], V[Ls].redirect()], ["wn", "b", "bp"], (right_channel, 0, 0))
    NR[Ls - 1] = unit([V[Ls], V[Ls].redirect()], ["b", "bp"], (0, 0))
    for j in range(Ls - 1, 0, -1):
        A, Ad = site(j, ["a", "s", "b"]), site(j, ["ap", "s", "bp"], True)
        t = A.contract(HR[j]).contract(M).contract(site(j, ["ap", "sp", "bp"], True))
        HR[j - 1] = relab(t, {"w": "wn", "a": "b", "ap": "bp"})
        NR[j - 1] = relab(A.contract(NR[j]).contract(Ad), {"a": "b", "ap": "bp"})
    hA, nA = [], []
    for k in range(Ls):
        Ak = site(k, ["a", "s", "b"])
        Y = HL[k].contract(Ak).contract(M).contract(HR[k])
        Y = Y.permute([Y.labels.index(l) for l in ("ap", "sp", "bp")])
        Z = NL[k].contract(Ak).contract(NR[k])
        Z = Z.permute([Z.labels.index(l) for l in ("ap", "s", "bp")])
        hA.append(_in_order(Y, Ak))
        nA.append(_in_order(Z, Ak))
    a0 = np.asarray(site_flats[0], np.float64)
    num = float(np.dot(a0, hA[0]))
    den = float(np.dot(a0, nA[0]))
    E = num / den
    grads = [(2.0 * h - 2.0 * E * n) / den for h, n in zip(hA, nA)]
    return num, den, grads


def _in_order(Y: BlockTensor, ref: BlockTensor) -> np.ndarray:
    """Y's blocks flattened in ref's block order (matched by qnum tuple)."""
    idx = {tuple(t): i for i, t in enumerate(Y.itoi.tolist())}
    return np.concatenate([Y.blocks[idx[tuple(t)]].ravel() for t in ref.itoi.tolist()])
