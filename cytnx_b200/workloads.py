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

from typing import Dict, List, Sequence, Tuple

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
        self.qv, self.dv = np.asarray(qv, np.int64), np.asarray(dv, np.int64)  # qv: [n] or [n][nsym]
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


def _qcol(q) -> np.ndarray:
    a = np.asarray(q, dtype=np.int64)
    return a.reshape(-1, 1) if a.ndim == 1 else a


def spec_bonds(spec: Spec):
    """(Vl, Vr, phys, inner) ket bonds of a two-site spec (one column per U(1) charge)."""
    from .core import BD_KET, Bond

    Vl = Bond(BD_KET, _qcol(spec.qv), spec.dv)
    Vr = Bond(BD_KET, _qcol(spec.qv_r), spec.dv_r)
    phys = Bond(BD_KET, _qcol(spec.phys_q), [1] * len(spec.phys_q))
    inner = Bond(BD_KET, _qcol(spec.inner_q), [1] * len(spec.inner_q))
    return Vl, Vr, phys, inner


def build_two_site(spec: Spec, mpo_vals, seed: int = 0, device=None, hermitian: bool = True):
    """Return (psi, L, M1, M2, R) cytnx_b200 UniTensors with the network leg order
    psi[a,s1,s2,b] L[w,a,a'] M[w,w',s,s'] R[w,b,b'], filled from a seeded generator."""
    from .core import BD_BRA, BD_KET, Bond
    from .unitensor import UniTensor
    import torch

    rng = np.random.default_rng(seed)
    Vl, Vr, phys, inner = spec_bonds(spec)
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


# ---------------------------------------------------------------- spinful Hubbard chain
# Site basis |0>, |up>, |dn>, |updn> = c+_up c+_dn |0>; charges (N, 2Sz).
HUB_PHYS_Q = [(0, 0), (1, 1), (1, -1), (2, 0)]
# MPO channels: 0 = identity (left), 1..4 = hopping pending after c+_up F, c+_dn F,
# c_up F, c_dn F, 5 = done; a channel's charge is q(w_in) + q(s) - q(s') of its opener.
HUB_INNER_Q = [(0, 0), (-1, -1), (-1, 1), (1, 1), (1, -1), (0, 0)]
HUB_P = [0, 3, 4, 1, 2, 5]


def hubbard_local_ops() -> Dict[str, np.ndarray]:
    """Site-local operators as matrices O[s', s] = <s'|O|s> (fermion order up before down)."""
    cu = np.zeros((4, 4))
    cu[0, 1] = 1.0   # c_up |up> = |0>
    cu[2, 3] = 1.0   # c_up c+_up c+_dn |0> = |dn>
    cd = np.zeros((4, 4))
    cd[0, 2] = 1.0   # c_dn |dn> = |0>
    cd[1, 3] = -1.0  # c_dn c+_up c+_dn |0> = -|up>
    F = np.diag([1.0, -1.0, -1.0, 1.0])
    return {"I": np.eye(4), "cu": cu, "cd": cd, "F": F, "nu": cu.T @ cu, "nd": cd.T @ cd}


def hubbard_mpo_values(U: float = 4.0, t: float = 1.0, mu: float = 0.0) -> Dict[Tuple[int, int, int, int], float]:
    """Nonzero entries M[w0, w1, s, s'] of the Hubbard MPO with Jordan-Wigner strings:
    H = -t sum_{i,sigma} (c+_{i,sigma} c_{i+1,sigma} + h.c.) + U sum_i n_up n_dn - mu sum_i n_i.
    The bond term c+_i c_{i+1} is (c+ F)_i (x) c_{i+1} and c+_{i+1} c_i = -(c F)_i (x) c+_{i+1}."""
    o = hubbard_local_ops()
    I, cu, cd, F, nu, nd = o["I"], o["cu"], o["cd"], o["F"], o["nu"], o["nd"]
    ops = {
        (0, 0): I, (5, 5): I,
        (0, 1): cu.T @ F, (1, 5): -t * cu,
        (0, 2): cd.T @ F, (2, 5): -t * cd,
        (0, 3): cu @ F, (3, 5): t * cu.T,
        (0, 4): cd @ F, (4, 5): t * cd.T,
        (0, 5): U * (nu @ nd) - mu * (nu + nd),
    }
    m = {}
    for (w0, w1), O in ops.items():
        for s in range(4):
            for sp in range(4):
                if O[sp, s] != 0.0:
                    m[(w0, w1, s, sp)] = float(O[sp, s])
    return m


def hubbard_sector_sizes(D: int, sigma: float = 4.0, center: Tuple[int, int] = (0, 0)):
    """Sectors (N, 2Sz) around ``center`` with weights exp(-dN^2/2s^2 - d(2Sz)^2/2s^2) on the
    lattice dN = d(2Sz) mod 2, sizes by largest remainder summing to D (empty ones dropped)."""
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


def hubbard_spec(D: int, sigma: float = 4.0) -> Spec:
    """Two-site Hubbard problem: left bond around (0, 0), right bond around (-2, 0) (two
    sites add N = 2 on average), both of dimension D."""
    ql, dl = hubbard_sector_sizes(D, sigma, (0, 0))
    qr, dr = hubbard_sector_sizes(D, sigma, (-2, 0))
    return Spec(ql, dl, HUB_PHYS_Q, HUB_INNER_Q, HUB_P, qr, dr)


def hubbard_batch_dims(nprob: int = 256, dmin: int = 128, dmax: int = 2048, seed: int = 0) -> List[int]:
    """Bond dimensions of the batched workload: D ~ U[dmin, dmax] (inclusive), seeded."""
    rng = np.random.default_rng(seed)
    return [int(d) for d in rng.integers(dmin, dmax + 1, size=nprob)]


def hubbard_mpo_unitensor(U: float = 4.0, t: float = 1.0, mu: float = 0.0, device=None):
    """The Hubbard MPO as a BlockUniTensor M[w_in (ket), w_out (bra), s (ket), s' (bra)] with
    (N, 2Sz) charges, and its (inner, phys) ket bonds."""
    from .core import BD_KET, Bond
    from .unitensor import UniTensor
    import torch

    phys = Bond(BD_KET, _qcol(HUB_PHYS_Q), [1] * 4)
    inner = Bond(BD_KET, _qcol(HUB_INNER_Q), [1] * 6)
    M = UniTensor([inner, inner.redirect(), phys, phys.redirect()], labels=["w0", "w1", "s", "sp"], rowrank=2,
                  device=device, name="MPO")
    mv = np.zeros(M._layout.nelem)
    idx = M._layout.index()
    for key, val in hubbard_mpo_values(U, t, mu).items():
        mv[M._layout.offs[idx[key]]] = val
    M._data.copy_(torch.from_numpy(mv))
    return M, inner, phys


def two_site_structure(spec: Spec, M):
    """Structure-only (L, M, M, R, psi) of a two-site problem (no device storage)."""
    from .unitensor import structure_only

    Vl, Vr, phys, inner = spec_bonds(spec)
    psi = structure_only([Vl, phys.redirect(), phys.redirect(), Vr.redirect()], ["a", "s1", "s2", "b"], 1)
    L = structure_only([inner.redirect(), Vl.redirect(), Vl], ["w", "a", "ap"], 1)
    R = structure_only([inner, Vr, Vr.redirect()], ["w", "b", "bp"], 1)
    return L, M, M, R, psi


def hubbard_batch(dims: Sequence[int], U: float = 4.0, t: float = 1.0, sigma: float = 4.0):
    """Structure-only two-site Hubbard problems, one per bond dimension in ``dims``."""
    from .core import Device

    M, _, _ = hubbard_mpo_unitensor(U, t, device=Device.cpu)
    return [two_site_structure(hubbard_spec(int(D), sigma), M) for D in dims]


def problem_data(problem, seed: int) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Seeded ~N(0,1) data of (L, R, psi) for a structure-only problem, rounded to FP32
    values (so FP32 and FP64 forms see the same numbers); psi is normalised."""
    L, _, _, R, psi = problem
    rng = np.random.default_rng(seed)
    l = rng.standard_normal(L._layout.nelem).astype(np.float32)
    r = rng.standard_normal(R._layout.nelem).astype(np.float32)
    x = rng.standard_normal(psi._layout.nelem)
    x = (x / np.linalg.norm(x)).astype(np.float32)
    return l, r, x


def materialize(u, flat, device=None):
    """A BlockUniTensor with the structure of ``u`` holding the flat data ``flat`` (FP64)."""
    from .core import Device
    from .unitensor import UniTensor
    import torch

    if device is None:
        dev = Device.torch_device(Device.cuda if torch.cuda.is_available() else Device.cpu)
    else:
        dev = device if isinstance(device, torch.device) else Device.torch_device(device)
    data = torch.as_tensor(np.asarray(flat, dtype=np.float64)).to(dev)
    return UniTensor._new_block(u.bonds(), u.labels(), u.rowrank(), u._layout, list(range(u.rank())), data)


def heff_network_lines() -> List[str]:
    """The two-site H_eff network of example/DMRG/dmrg_two_sites_U1.py:29-34."""
    return ["psi: -1,-2,-3,-4", "L: -5,-1,0", "R: -7,-4,3", "M1: -5,-6,-2,1", "M2: -6,-7,-3,2", "TOUT: 0,1;2,3"]
