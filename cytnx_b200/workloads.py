"""Seeded synthetic DMRG problems (the benchmark configurations).

* ``u1_sector_sizes(D, qmax=16, var=72)``: sector sizes proportional to exp(-q^2/var) for
  q = -qmax..qmax, rounded by largest remainder so they sum to D.
* ``xxz_mpo(Jz, Jxy, h)``: the exact spin-1/2 XXZ MPO, bond dimension 5, physical
  charges +-1 (2 Sz), inner channel charges [0, -2, +2, 0, 0] (I, S+ then S-, S- then S+,
  Sz, I) in the leg convention of example/DMRG/dmrg_two_sites_U1.py:43-60
  (M[w_in KET, w_out BRA, s KET, s' BRA] = coefficient * <s'|O|s>).
* ``random_env`` / ``random_psi``: ~N(0,1) data in every symmetry-allowed block of the
  environments L[w,a,a'], R[w,b,b'] (made Hermitian: L[w,a,a'] = L[P w,a',a] with P the
  channel conjugation 1<->2, same for R) and the two-site wavefunction psi[a,s1,s2,b].

Data are generated on the host with numpy's PCG64 (seeded) and shared by the GPU path
and the CPU oracle; no reference RNG stream is reproduced.
"""
from __future__ import annotations

from typing import Dict, List, Tuple

import numpy as np

SQRT_HALF = np.sqrt(0.5)


def u1_sector_sizes(D: int, qmax: int = 16, var: float = 72.0) -> Tuple[np.ndarray, np.ndarray]:
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


class Spec:
    """Bond tables of the two-site problem (host-side, numpy)."""

    def __init__(self, qv: np.ndarray, dv: np.ndarray, phys_q: List[int], inner_q: List[int], P: List[int],
                 qv_r: np.ndarray = None, dv_r: np.ndarray = None):
        self.qv, self.dv = np.asarray(qv, np.int64), np.asarray(dv, np.int64)
        self.qv_r = self.qv if qv_r is None else np.asarray(qv_r, np.int64)
        self.dv_r = self.dv if dv_r is None else np.asarray(dv_r, np.int64)
        self.phys_q = list(phys_q)
        self.inner_q = list(inner_q)
        self.P = list(P)  # channel conjugation


def xxz_mpo_values(Jz: float = 1.0, Jxy: float = 1.0, h: float = 0.0) -> Dict[Tuple[int, int, int, int], float]:
    """Nonzero entries M[w0, w1, s, s'] (s index 0 = up (+1), 1 = down (-1))."""
    c = np.sqrt(abs(Jxy) / 2.0)
    sz = {0: 0.5, 1: -0.5}
    m = {}
    for s in (0, 1):
        m[(0, 0, s, s)] = 1.0
        m[(4, 4, s, s)] = 1.0
        m[(0, 3, s, s)] = sz[s]
        m[(3, 4, s, s)] = Jz * sz[s]
        if h:
            m[(0, 4, s, s)] = h * sz[s]
    sgn = 1.0 if Jxy >= 0 else -1.0
    m[(0, 1, 1, 0)] = c          # S+ : <up|S+|down> = 1
    m[(1, 4, 0, 1)] = sgn * c    # S- : <down|S-|up> = 1
    m[(0, 2, 0, 1)] = c          # S-
    m[(2, 4, 1, 0)] = sgn * c    # S+
    return m


XXZ_INNER_Q = [0, -2, 2, 0, 0]
XXZ_P = [0, 2, 1, 3, 4]
SPIN_PHYS_Q = [1, -1]


def xxz_spec(D: int, qmax: int = 16, var: float = 72.0) -> Spec:
    qv, dv = u1_sector_sizes(D, qmax, var)
    return Spec(qv, dv, SPIN_PHYS_Q, XXZ_INNER_Q, XXZ_P)


def build_two_site(spec: Spec, mpo_vals, seed: int = 0, device=None, hermitian: bool = True):
    """Return (psi, L, M1, M2, R) cytnx_b200 UniTensors with the network leg order
    psi[a,s1,s2,b] L[w,a,a'] M[w,w',s,s'] R[w,b,b'], filled from a seeded generator."""
    from .core import BD_BRA, BD_KET, Bond
    from .unitensor import UniTensor
    import torch

    rng = np.random.default_rng(seed)
    Vl = Bond(BD_KET, spec.qv.reshape(-1, 1), spec.dv)
    Vr = Bond(BD_KET, spec.qv_r.reshape(-1, 1), spec.dv_r)
    phys = Bond(BD_KET, np.array(spec.phys_q).reshape(-1, 1), [1] * len(spec.phys_q))
    inner = Bond(BD_KET, np.array(spec.inner_q).reshape(-1, 1), [1] * len(spec.inner_q))
    psi = UniTensor([Vl, phys.redirect(), phys.redirect(), Vr.redirect()], labels=["a", "s1", "s2", "b"],
                    rowrank=1, device=device, name="psi")
    L = UniTensor([inner.redirect(), Vl.redirect(), Vl], labels=["w", "a", "ap"], rowrank=1, device=device, name="L")
    R = UniTensor([inner, Vr, Vr.redirect()], labels=["w", "b", "bp"], rowrank=1, device=device, name="R")
    M = UniTensor([inner, inner.redirect(), phys, phys.redirect()], labels=["w0", "w1", "s", "sp"], rowrank=2,
                  device=device, name="MPO")
    # MPO values (host -> device once)
    mv = np.zeros(M._layout.nelem)
    idx = M._layout.index()
    for key, val in mpo_vals.items():
        b = idx.get(key)
        if b is None:
            raise ValueError(f"MPO entry {key} violates the symmetry")
        mv[M._layout.offs[b]] = val
    M._data.copy_(torch.from_numpy(mv))

    def fill_env(U, P):
        lay = U._layout
        data = rng.standard_normal(lay.nelem)
        if hermitian:
            sym = data.copy()
            ix = lay.index()
            for b, (w, x, y) in enumerate(lay.itoi.tolist()):
                b2 = ix[(P[w], y, x)]
                o1, o2 = lay.offs[b], lay.offs[b2]
                s1 = lay.shapes[b]
                A = data[o1: o1 + lay.sizes[b]].reshape(s1)
                Bt = data[o2: o2 + lay.sizes[b2]].reshape(lay.shapes[b2])
                sym[o1: o1 + lay.sizes[b]] = (0.5 * (A + Bt.transpose(0, 2, 1))).reshape(-1)
            data = sym
        U._data.copy_(torch.from_numpy(data))

    fill_env(L, spec.P)
    fill_env(R, spec.P)
    x = rng.standard_normal(psi._layout.nelem)
    x /= np.linalg.norm(x)
    psi._data.copy_(torch.from_numpy(x))
    M2 = M.clone().set_name_("MPO2")
    return psi, L, M, M2, R


def xxz_mpo_unitensor(Jz: float = 1.0, Jxy: float = 1.0, h: float = 0.0, device=None):
    """The XXZ MPO as a BlockUniTensor M[w_in (ket), w_out (bra), s (ket), s' (bra)] and its bonds."""
    from .core import BD_KET, Bond
    from .unitensor import UniTensor
    import torch

    phys = Bond(BD_KET, np.array(SPIN_PHYS_Q).reshape(-1, 1), [1, 1])
    inner = Bond(BD_KET, np.array(XXZ_INNER_Q).reshape(-1, 1), [1] * 5)
    M = UniTensor([inner, inner.redirect(), phys, phys.redirect()], labels=["w0", "w1", "s", "sp"], rowrank=2,
                  device=device, name="MPO")
    mv = np.zeros(M._layout.nelem)
    idx = M._layout.index()
    for key, val in xxz_mpo_values(Jz, Jxy, h).items():
        mv[M._layout.offs[idx[key]]] = val
    M._data.copy_(torch.from_numpy(mv))
    return M, inner, phys


def heff_network_lines() -> List[str]:
    """The two-site H_eff network of example/DMRG/dmrg_two_sites_U1.py:29-34."""
    return ["psi: -1,-2,-3,-4", "L: -5,-1,0", "R: -7,-4,3", "M1: -5,-6,-2,1", "M2: -6,-7,-3,2", "TOUT: 0,1;2,3"]
