"""Block SVD and its truncation (the step after Lanczos in two-site DMRG).

Follows ``linalg::Gesvd`` / ``linalg::Svd_truncate`` for BlockUniTensor
(src/linalg/Svd.cpp:193-, src/linalg/Svd_truncate.cpp:154-340): blocks are grouped by
the total charge of the row legs (rowrank), each charge sector is assembled into one
matrix (row-leg block combinations x column-leg block combinations), decomposed, and the
singular values of all sectors are sorted together; truncation keeps the largest
``keepdim`` values (an exact degeneracy at the cut is kept whole, values below ``err``
are dropped, at least ``mindim`` are kept) and removes sectors that keep nothing.

Outputs: U [row legs..., "_aux_L" (bra)], S ["_aux_L" (ket), "_aux_R" (bra)],
vT ["_aux_R" (ket), column legs...].  S is returned with square diagonal blocks (a
BlockUniTensor whose blocks are diag(s)); its norm, scaling and contraction behave as
the reference's diagonal tensor.  The per-sector decompositions use the device's
LAPACK-class library (torch.linalg.svd -> cuSOLVER): this row is off the hot path.
"""
from __future__ import annotations

from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from ._lib import CytnxError
from .core import BD_BRA, BD_KET, Bond, Symmetry, Tensor, Type
from .unitensor import UniTensor, UTenType, layout_for


def _row_charge(u: UniTensor, tup: Sequence[int]) -> Tuple[int, ...]:
    syms = u.syms()
    q = []
    for s_i, sym in enumerate(syms):
        tot = 0
        first = True
        for leg in range(u.rowrank()):
            b = u._bonds[leg]
            v = int(b._qnums[tup[leg], s_i])
            if b.type() == BD_BRA:
                v = sym.reverse_rule(v)
            tot = v if first else sym.combine_rule(tot, v)
            first = False
        q.append(tot)
    return tuple(q)


def _sectors(u: UniTensor):
    """Group the blocks of a contiguous BlockUniTensor by row charge: sectors in ascending
    charge order, rows and columns of a sector in ascending qindex-tuple order (the std::map
    and vec_sort orders of Gesvd_BlockUT_internal, src/linalg/Gesvd.cpp:238-262)."""
    r = u.rowrank()
    itoi = u._layout.itoi.tolist()
    sec: Dict[tuple, dict] = {}
    for b, t in enumerate(itoi):
        q = _row_charge(u, t)
        s = sec.setdefault(q, {"rows": set(), "cols": set(), "blocks": []})
        rt, ct = tuple(t[:r]), tuple(t[r:])
        s["rows"].add(rt)
        s["cols"].add(ct)
        s["blocks"].append((b, rt, ct))
    order = sorted(sec)
    for q in order:
        sec[q]["rows"] = sorted(sec[q]["rows"])
        sec[q]["cols"] = sorted(sec[q]["cols"])
    return order, sec


def _deg(u: UniTensor, legs: Sequence[int], tup: Sequence[int]) -> int:
    d = 1
    for leg, q in zip(legs, tup):
        d *= int(u._bonds[leg]._degs[q])
    return d


def _svd_blocks(u: UniTensor):
    if u.uten_type() != UTenType.Block:
        raise CytnxError("[Svd] this path handles BlockUniTensors; dense tensors use torch.linalg.svd directly")
    u = u.contiguous()
    r = u.rowrank()
    if r <= 0 or r >= u.rank():
        raise CytnxError("[Svd] rowrank must split the legs (0 < rowrank < rank)")
    rl, cl = list(range(r)), list(range(r, u.rank()))
    order, sec = _sectors(u)
    out = []
    for q in order:
        s = sec[q]
        rd = [_deg(u, rl, rt) for rt in s["rows"]]
        cd = [_deg(u, cl, ct) for ct in s["cols"]]
        ro = np.concatenate([[0], np.cumsum(rd)]).astype(int)
        co = np.concatenate([[0], np.cumsum(cd)]).astype(int)
        M = torch.zeros(int(ro[-1]), int(co[-1]), dtype=u._data.dtype, device=u._data.device)
        for b, rt, ct in s["blocks"]:
            i, j = s["rows"].index(rt), s["cols"].index(ct)
            off, sz = int(u._layout.offs[b]), int(u._layout.sizes[b])
            M[ro[i]:ro[i + 1], co[j]:co[j + 1]] = u._data[off:off + sz].view(rd[i], cd[j])
        U, S, Vh = torch.linalg.svd(M, full_matrices=False)
        out.append((q, s, rd, cd, ro, co, U, S, Vh))
    return u, out


def _assemble(u: UniTensor, parts, keep: List[int], is_U: bool, is_vT: bool):
    r = u.rowrank()
    syms = u.syms()
    kept = [(p, k) for p, k in zip(parts, keep) if k > 0]
    qn = np.array([list(p[0]) for p, _ in kept], dtype=np.int64).reshape(len(kept), len(syms))
    degs = [k for _, k in kept]
    new_bra = Bond(BD_BRA, qn, degs, syms)
    new_ket = Bond(BD_KET, qn, degs, syms)
    dev = u._data.device
    dt = Type.from_torch(u._data.dtype)
    # S with square diagonal blocks
    S = UniTensor([new_ket, new_bra], labels=["_aux_L", "_aux_R"], rowrank=1, dtype=dt, device=u.device())
    sidx = S._layout.index()
    for qi, ((q, s, rd, cd, ro, co, Um, Sv, Vh), k) in enumerate(kept):
        b = sidx[(qi, qi)]
        off = int(S._layout.offs[b])
        S._data[off:off + k * k] = torch.diag(Sv[:k]).reshape(-1)
    res = [S]
    if is_U:
        Ut = UniTensor([b.clone() for b in u._bonds[:r]] + [new_bra], labels=u.labels()[:r] + ["_aux_L"],
                       rowrank=r, dtype=dt, device=u.device())
        ui = Ut._layout.index()
        for qi, ((q, s, rd, cd, ro, co, Um, Sv, Vh), k) in enumerate(kept):
            for i, rt in enumerate(s["rows"]):
                b = ui.get(tuple(rt) + (qi,))
                if b is None:
                    continue
                off, sz = int(Ut._layout.offs[b]), int(Ut._layout.sizes[b])
                Ut._data[off:off + sz] = Um[ro[i]:ro[i + 1], :k].reshape(-1)
        res.append(Ut)
    if is_vT:
        Vt = UniTensor([new_ket] + [b.clone() for b in u._bonds[r:]], labels=["_aux_R"] + u.labels()[r:], rowrank=1,
                       dtype=dt, device=u.device())
        vi = Vt._layout.index()
        for qi, ((q, s, rd, cd, ro, co, Um, Sv, Vh), k) in enumerate(kept):
            for j, ct in enumerate(s["cols"]):
                b = vi.get((qi,) + tuple(ct))
                if b is None:
                    continue
                off, sz = int(Vt._layout.offs[b]), int(Vt._layout.sizes[b])
                Vt._data[off:off + sz] = Vh[:k, co[j]:co[j + 1]].reshape(-1)
        res.append(Vt)
    return res


def Gesvd(Tin: UniTensor, is_U: bool = True, is_vT: bool = True) -> List[UniTensor]:
    """[S, U, vT] (U / vT omitted when not requested) of a BlockUniTensor."""
    u, parts = _svd_blocks(Tin)
    keep = [int(p[7].numel()) for p in parts]
    return _assemble(u, parts, keep, is_U, is_vT)


Svd = Gesvd


def _cut(Sall: np.ndarray, keep_dim: int, err: float, floor: int):
    """Cut value Smin on ascending singular values: keep_dim from the top, raised past values
    below err while more than `floor` stay (Svd_truncate.cpp:166-191); None keeps nothing."""
    n = len(Sall)
    if keep_dim < n:
        smidx = n - keep_dim
    else:
        keep_dim, smidx = n, 0
    smin = Sall[smidx]
    while smin < err and keep_dim > floor:
        keep_dim -= 1
        if keep_dim == 0:
            return None
        smidx += 1
        smin = Sall[smidx]
    return smin


def Gesvd_truncate(Tin: UniTensor, keepdim: int, *args, err: float = 0.0, is_U: bool = True, is_vT: bool = True,
                   return_err: int = 0, mindim: int = 1, min_blockdim=None):
    """linalg::Gesvd_truncate (src/linalg/Gesvd_truncate.cpp): ``Gesvd_truncate(T, keepdim, err,
    is_U, is_vT, return_err, mindim)`` or, with a per-sector floor, ``Gesvd_truncate(T, keepdim,
    min_blockdim, err, is_U, is_vT, return_err, mindim)`` (:430-560): the first min_blockdim[b]
    values of sector b are kept outside the global ranking (one entry applies to every sector)."""
    args = list(args)
    if args and isinstance(args[0], (list, tuple, np.ndarray)):
        min_blockdim = list(args.pop(0))
    names = ["err", "is_U", "is_vT", "return_err", "mindim"]
    vals = dict(err=err, is_U=is_U, is_vT=is_vT, return_err=return_err, mindim=mindim)
    for n_, v in zip(names, args):
        vals[n_] = v
    err, is_U, is_vT, return_err, mindim = (vals[n_] for n_ in names)
    if min_blockdim is None:
        res = Svd_truncate(Tin, keepdim, err, True, return_err, mindim)
        S, U, Vt = res[:3]
        out = [S] + ([U] if is_U else []) + ([Vt] if is_vT else [])
        return out + res[3:]
    u, parts = _svd_blocks(Tin)
    nb = len(parts)
    mb = [int(x) for x in min_blockdim]
    if len(mb) == 1:
        mb = mb * nb
    if len(mb) != nb:
        raise CytnxError("[ERROR][Gesvd_truncate] min_blockdim must have the same number of elements as blocks "
                         "in the singular value UniTensor")
    keep_dim, min_dim = int(keepdim), max(1, int(mindim))
    rest, any_mb = [], False
    for b, p in enumerate(parts):
        v = p[7].cpu().numpy()
        if mb[b] < 1:
            rest.append(v)
            continue
        any_mb = True
        if len(v) <= mb[b]:
            keep_dim -= len(v)
            min_dim -= len(v)
            continue
        rest.append(v[mb[b]:])
        keep_dim -= mb[b]
        min_dim -= mb[b]
    smin = None
    Srest = np.sort(np.concatenate(rest)) if rest else np.zeros(0)
    if rest and keep_dim > 0:
        min_dim = max(1, min_dim) if not any_mb else max(0, min_dim)
        smin = _cut(Srest, keep_dim, err, min_dim)
    keep = []
    for b, p in enumerate(parts):
        v = p[7].cpu().numpy()
        k = min(mb[b], len(v))
        if smin is not None:
            above = np.nonzero(v[mb[b]:] >= smin)[0]
            if len(above):
                k = mb[b] + int(above[-1]) + 1
        keep.append(k)
    res = _assemble(u, parts, keep, is_U, is_vT)
    if return_err:
        dropped = np.sort(np.concatenate([p[7].cpu().numpy()[k:] for p, k in zip(parts, keep)])) \
            if parts else np.zeros(0)
        e = float(dropped.max()) if return_err == 1 and len(dropped) else 0.0
        res.append(Tensor.from_numpy(np.array([e]), -1) if return_err == 1 else Tensor.from_numpy(dropped[::-1], -1))
    return res


def Svd_truncate(Tin: UniTensor, keepdim: int, err: float = 0.0, is_UvT: bool = True, return_err: int = 0,
                 mindim: int = 1):
    """Truncated block SVD keeping the ``keepdim`` largest singular values overall."""
    u, parts = _svd_blocks(Tin)
    allS = torch.cat([p[7] for p in parts]) if parts else torch.zeros(0)
    Sall = torch.sort(allS).values.cpu().numpy()  # ascending, as Svd_truncate.cpp:166-191
    n = len(Sall)
    keep_dim = int(keepdim)
    if keep_dim < n:
        smidx = n - keep_dim
    else:
        keep_dim, smidx = n, 0
    Smin = Sall[smidx] if n else 0.0
    while Smin < err and keep_dim > max(1, mindim):
        keep_dim -= 1
        smidx += 1
        Smin = Sall[smidx]
    keep = [int((p[7] >= float(Smin)).sum().item()) for p in parts]
    # an exact degeneracy at the cut stays whole (values >= Smin are kept)
    res = _assemble(u, parts, keep, is_UvT, is_UvT)
    if return_err:
        dropped = Sall[:n - sum(keep)]
        e = float(dropped.max()) if return_err == 1 and len(dropped) else 0.0
        res.append(Tensor.from_numpy(np.array([e]), -1) if return_err == 1 else Tensor.from_numpy(dropped, -1))
    return res
