"""Reverse-mode differentiation of block-sparse contractions, and a differentiable
U(1) MPS energy built on it.

``ContractFn`` is a ``torch.autograd.Function`` around ``Contract`` of two
BlockUniTensors whose storages are plain torch tensors (the flat block buffers are
torch storage already, so nothing is copied in or out).  Its backward is written by
hand: for C = sum_comm A B,

    dA = Contract(dC, B~)   and   dB = Contract(A~, dC)

where X~ is X with every bond redirected (same blocks, same storage: a real tensor's
adjoint under the flux rule), followed by a permutation back to the operand's storage
order.  Both products run on the CUDA contraction engine, so the backward pass costs
two forward-sized contractions and nothing falls back to generic autograd.

``mps_energy`` evaluates E = <A|H|A> / <A|A> for a finite MPS by a left-to-right sweep
of environments (H: L[w,a,a'], norm: N[a,a']); with ``checkpoint_every = k`` the sweep
is cut into segments of k sites under ``torch.utils.checkpoint``, so only every k-th
environment stays resident and the others are recomputed in the backward pass.

The environment recursions are those of the reference's DMRG example
(example/DMRG/dmrg_two_sites_U1.py:63-85, L' = L A M A^dagger), built with Contract.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch
from torch.utils.checkpoint import checkpoint

from ._lib import CytnxError
from .core import BD_BRA, BD_KET, Bond
from .unitensor import Contract, UniTensor, UTenType


class Struct:
    """Metadata of a BlockUniTensor without its storage (bonds, labels, layout, mapper)."""

    __slots__ = ("bonds", "labels", "rowrank", "layout", "mapper")

    def __init__(self, bonds, labels, rowrank, layout, mapper):
        self.bonds, self.labels, self.rowrank, self.layout, self.mapper = bonds, labels, rowrank, layout, mapper

    @classmethod
    def of(cls, u: UniTensor) -> "Struct":
        if u.uten_type() != UTenType.Block:
            raise CytnxError("[autodiff] operands must be BlockUniTensors")
        return cls(list(u._bonds), list(u._labels), u._rowrank, u._layout, list(u._mapper))

    def wrap(self, data: torch.Tensor) -> UniTensor:
        return UniTensor._new_block(self.bonds, self.labels, self.rowrank, self.layout, self.mapper, data)

    def physical_labels(self) -> List[str]:
        ph = [None] * len(self.labels)
        for i, m in enumerate(self.mapper):
            ph[m] = self.labels[i]
        return ph

    def relabel(self, labels: Sequence[str]) -> "Struct":
        return Struct(self.bonds, [str(l) for l in labels], self.rowrank, self.layout, self.mapper)

    def dagger(self) -> "Struct":
        """Struct of the Dagger of a real tensor: bonds redirected, legs reversed, same storage."""
        r = len(self.bonds)
        rev = list(range(r - 1, -1, -1))
        return Struct([self.bonds[i].redirect() for i in rev], [self.labels[i] for i in rev], r - self.rowrank,
                      self.layout, [self.mapper[i] for i in rev])


def redirect_all(u: UniTensor) -> UniTensor:
    """Every bond redirected; redirected bonds enumerate the same blocks, so the storage
    and its layout are shared."""
    v = u.clone_meta()
    v._bonds = [b.redirect() for b in u._bonds]
    v._is_braket = v._update_braket()
    return v


def _to_storage(g: UniTensor, s: Struct) -> torch.Tensor:
    """A gradient with the logical legs of ``s`` laid out like the storage of ``s``."""
    gp = g.permute(s.physical_labels()).contiguous()
    lay = gp._layout
    if lay is not s.layout and not (lay.nelem == s.layout.nelem and np.array_equal(lay.itoi, s.layout.itoi)):
        raise CytnxError("[autodiff] gradient block structure differs from the operand's")
    return gp._data


class ContractFn(torch.autograd.Function):
    """C = Contract(A, B) on flat storages ``a`` / ``b`` described by ``sa`` / ``sb``;
    returns C's flat storage (its Struct is left in ``ContractFn.last_struct``)."""

    last_struct: Optional[Struct] = None

    @staticmethod
    def forward(ctx, a, b, sa: Struct, sb: Struct):
        C = Contract(sa.wrap(a), sb.wrap(b))
        if C.uten_type() != UTenType.Block:
            raise CytnxError("[autodiff] full contractions (scalar results) are taken with torch.dot instead")
        ctx.save_for_backward(a, b)
        ctx.sa, ctx.sb = sa, sb
        ctx.sc = Struct.of(C)
        ContractFn.last_struct = ctx.sc
        return C._data

    @staticmethod
    def backward(ctx, gc):
        a, b = ctx.saved_tensors
        G = ctx.sc.wrap(gc.contiguous())
        ga = gb = None
        if ctx.needs_input_grad[0]:
            ga = _to_storage(Contract(G, redirect_all(ctx.sb.wrap(b))), ctx.sa)
        if ctx.needs_input_grad[1]:
            gb = _to_storage(Contract(redirect_all(ctx.sa.wrap(a)), G), ctx.sb)
        return ga, gb, None, None


def contract(a: torch.Tensor, sa: Struct, b: torch.Tensor, sb: Struct) -> Tuple[torch.Tensor, Struct]:
    """Differentiable Contract on flat storages; returns (storage, Struct) of the result."""
    out = ContractFn.apply(a, b, sa, sb)
    return out, ContractFn.last_struct


# ---------------------------------------------------------------- U(1) MPS
def mps_bond_sectors(L: int, k: int, Dmax: int) -> Tuple[np.ndarray, np.ndarray]:
    """Charges and sizes of bond k (after k sites) of a total-Sz = 0 spin-1/2 MPS: charge
    q = -(sum of 2Sz of the left k sites); each sector is capped by the number of states
    of either side with that charge, the bond by Dmax, sizes proportional to the caps."""
    from math import comb

    qs, caps = [], []
    for q in range(-k, k + 1, 2):
        nl = (k - q) // 2
        nr = (L - k + q) // 2
        if not (0 <= nl <= k and 0 <= nr <= L - k) or (L - k + q) % 2:
            continue
        c = min(comb(k, nl), comb(L - k, nr))
        if c > 0:
            qs.append(q)
            caps.append(c)
    caps = np.array(caps, dtype=np.float64)
    D = int(min(Dmax, caps.sum()))
    raw = D * caps / caps.sum()
    base = np.floor(raw).astype(np.int64)
    rem = D - int(base.sum())
    order = sorted(range(len(qs)), key=lambda i: (-(raw[i] - base[i]), abs(qs[i]), qs[i]))
    for i in order[:rem]:
        base[i] += 1
    base = np.minimum(base, caps.astype(np.int64))
    keep = base > 0
    return np.array(qs, dtype=np.int64)[keep], base[keep]


class U1MPS:
    """A finite spin-1/2 MPS with U(1) (2Sz) blocks, total Sz = 0, and the XXZ MPO.

    Site k holds A_k[a (ket), s (bra), b (bra)] with flux q_a - q_s - q_b = 0; its
    storage is a flat float64 tensor ``params[k]`` (a leaf for autograd)."""

    def __init__(self, L: int, Dmax: int, seed: int = 0, Jz: float = 1.0, Jxy: float = 1.0, h: float = 0.0,
                 device=None):
        from .workloads import xxz_mpo_unitensor

        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.L, self.Dmax, self.device = L, Dmax, device
        self.M, inner, phys = xxz_mpo_unitensor(Jz, Jxy, h, device=device.index if device.type == "cuda" else -1)
        self.inner, self.phys = inner, phys
        bonds = []
        for k in range(L + 1):
            q, d = mps_bond_sectors(L, k, Dmax)
            bonds.append(Bond(BD_KET, q.reshape(-1, 1), d))
        self.bonds = bonds
        rng = np.random.default_rng(seed)
        self.structs: List[Struct] = []
        self.params: List[torch.Tensor] = []
        for k in range(L):
            u = UniTensor([bonds[k], phys.redirect(), bonds[k + 1].redirect()], labels=["a", "s", "b"], rowrank=2,
                          device=device.index if device.type == "cuda" else -1)
            s = Struct.of(u)
            sigma = 1.0 / np.sqrt(2.0 * bonds[k].dim())
            x = torch.from_numpy(rng.standard_normal(u._layout.nelem) * sigma).to(device)
            self.structs.append(s)
            self.params.append(x.requires_grad_(True))
        # boundary environments: H channel 0 on the left, channel 4 closes on the right
        v0 = bonds[0]
        Lb = UniTensor([inner.redirect(), v0.redirect(), v0], labels=["w", "a", "ap"], rowrank=1,
                       device=device.index if device.type == "cuda" else -1)
        Lb.set_elem([0, 0, 0], 1.0)
        Nb = UniTensor([v0.redirect(), v0], labels=["a", "ap"], rowrank=1,
                       device=device.index if device.type == "cuda" else -1)
        Nb.set_elem([0, 0], 1.0)
        self.Lb, self.Nb = Lb, Nb
        self.sM = Struct.of(self.M.relabel(["w", "wn", "s", "sp"]))

    def numel(self) -> int:
        return sum(int(p.numel()) for p in self.params)

    # ---------------------------------------------------------------- environments
    def _site_step(self, Ld, sL: Struct, Nd, sN: Struct, x, sA: Struct):
        """One site of the left sweep: L' = L A M A^dagger, N' = N A A^dagger."""
        sAd = sA.dagger().relabel(["bp", "sp", "ap"])  # Dagger of A[a,s,b] is A*[b,s,a]
        t, st = contract(Ld, sL, x, sA)                   # (w, ap, s, b)
        t, st = contract(t, st, self.M._data, self.sM)    # (ap, b, wn, sp)
        t, st = contract(t, st, x, sAd)                   # (b, wn, bp)
        sL2 = st.relabel([{"b": "a", "wn": "w", "bp": "ap"}[l] for l in st.labels])
        u, su = contract(Nd, sN, x, sA)                   # (ap, s, b)
        u, su = contract(u, su, x, sAd.relabel(["bp", "s", "ap"]))  # (b, bp)
        sN2 = su.relabel([{"b": "a", "bp": "ap"}[l] for l in su.labels])
        return t, sL2, u, sN2

    def energy(self, params: Optional[Sequence[torch.Tensor]] = None, checkpoint_every: int = 4,
               numerator_only: bool = False) -> torch.Tensor:
        """E = <A|H|A> / <A|A> (or <A|H|A> with ``numerator_only``), differentiable in params."""
        params = self.params if params is None else params
        Ld, sL = self.Lb._data, Struct.of(self.Lb)
        Nd, sN = self.Nb._data, Struct.of(self.Nb)
        k = 0
        while k < self.L:
            seg = list(range(k, min(self.L, k + max(1, checkpoint_every))))
            if checkpoint_every and checkpoint_every > 0 and torch.is_grad_enabled():
                structs_out = {}

                def run(Ld_, Nd_, *xs, seg=seg, sL=sL, sN=sN, structs_out=structs_out):
                    l, sl, n, sn = Ld_, sL, Nd_, sN
                    for j, x in zip(seg, xs):
                        l, sl, n, sn = self._site_step(l, sl, n, sn, x, self.structs[j])
                    structs_out["L"], structs_out["N"] = sl, sn
                    return l, n

                Ld, Nd = checkpoint(run, Ld, Nd, *[params[j] for j in seg], use_reentrant=False)
                sL, sN = structs_out["L"], structs_out["N"]
            else:
                for j in seg:
                    Ld, sL, Nd, sN = self._site_step(Ld, sL, Nd, sN, params[j], self.structs[j])
            k = seg[-1] + 1
        # closing: H channel 4 of L_L[w, a, a'] (a, a' one-dimensional), N_L[0, 0]
        wl = sL.labels.index("w")
        itoi = sL.layout.itoi
        hit = [b for b in range(len(itoi)) if int(itoi[b][sL.mapper[wl]]) == 4]
        if len(hit) != 1:
            raise CytnxError("[U1MPS.energy] closing channel not found")
        num = Ld[int(sL.layout.offs[hit[0]])]
        if numerator_only:
            return num
        den = Nd[0]
        return num / den

    # ---------------------------------------------------------------- effective Hamiltonian (no autograd)
    def heff_times_site(self, k: int) -> torch.Tensor:
        """(H_eff,k A_k) in A_k's storage layout, from environments built with Contract."""
        with torch.no_grad():
            A = [self.structs[j].wrap(self.params[j].detach()) for j in range(self.L)]
            Mr = self.M.relabel(["w", "wn", "s", "sp"])
            Lenv = self.Lb
            for j in range(k):
                Aj = A[j].relabel(["a", "s", "b"])
                Ad = Aj.Dagger().relabel(["bp", "sp", "ap"])
                Lenv = Contract(Contract(Contract(Lenv, Aj), Mr), Ad)
                Lenv = Lenv.relabel([{"b": "a", "wn": "w", "bp": "ap"}[l] for l in Lenv.labels()])
            vL = self.bonds[self.L]
            Renv = UniTensor([self.inner, vL, vL.redirect()], labels=["wn", "b", "bp"], rowrank=1,
                             device=self.device.index if self.device.type == "cuda" else -1)
            Renv.set_elem([4, 0, 0], 1.0)
            Mr2 = self.M.relabel(["w", "wn", "s", "sp"])
            for j in range(self.L - 1, k, -1):
                Aj = A[j].relabel(["a", "s", "b"])
                Ad = Aj.Dagger().relabel(["bp", "sp", "ap"])
                Renv = Contract(Contract(Contract(Aj, Renv), Mr2), Ad)   # (w, a, ap)
                Renv = Renv.relabel([{"w": "wn", "a": "b", "ap": "bp"}[l] for l in Renv.labels()])
            Ak = A[k].relabel(["a", "s", "b"])
            Y = Contract(Contract(Contract(Lenv, Ak), Mr), Renv)           # (ap, sp, bp)
            Y = Y.relabel([{"ap": "a", "sp": "s", "bp": "b"}[l] for l in Y.labels()])
            return _to_storage(Y, self.structs[k].relabel(["a", "s", "b"]))
