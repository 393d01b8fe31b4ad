"""Block SVD and its truncation on the CPU -- TEST INFRASTRUCTURE, never part of the product.

Restates, on ``oracle.BlockTensor`` with numpy's LAPACK:

* ``gesvd``           -- ``Gesvd_BlockUT_internal`` (src/linalg/Gesvd.cpp:191-330): blocks grouped by
                         the total charge of the row legs (row-leg charges in the KET frame, summed);
                         sectors in ascending charge order (the std::map key order); inside a sector
                         the blocks sorted by (row qindex tuple, column qindex tuple) and glued into
                         one matrix; one SVD per sector.  S is the diagonal of "_aux_L" (KET) x
                         "_aux_R" (BRA), U = row legs + "_aux_L" (BRA), vT = "_aux_R" (KET) + column legs.
* ``svd_truncate``    -- ``Svd_truncate_Block_UTs_internal`` (src/linalg/Svd_truncate.cpp:153-301):
                         all singular values sorted ascending, the cut value Smin at keepdim from the
                         top (raised past values below ``err`` while more than max(1, mindim) stay),
                         every value >= Smin kept, sectors that keep nothing removed.
* ``gesvd_truncate``  -- ``Gesvd_truncate_Block_UTs_internal`` with ``min_blockdim``
                         (src/linalg/Gesvd_truncate.cpp:430-560): the first min_blockdim[b] values of
                         each sector are kept outside the global ranking.

Only what the tests compare is built: per-sector singular values and U / vT blocks.
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence

import numpy as np

from . import Bond, BlockTensor, enumerate_blocks


def _row_charge(T: BlockTensor, tup) -> tuple:
    r = T.rowrank
    q = None
    for leg in range(r):
        b = T.bonds[leg]
        v = b.qnums[tup[leg]].copy()
        if b.type == 1:  # BRA legs enter reversed (U1: negated; Zn: n - q)
            v = np.array([(s[1] - x) % s[1] if s[0] == 0 else -x for x, s in zip(v, b.syms)])
        q = v if q is None else np.array([(a + c) % s[1] if s[0] == 0 else a + c
                                          for a, c, s in zip(q, v, b.syms)])
    return tuple(int(x) for x in q)


class BlockSvd:
    """Per-sector SVD of a BlockTensor: ``charges`` (ascending), and for each sector the row /
    column qindex tuples, their sizes, and U, s, Vh."""

    def __init__(self, T: BlockTensor):
        r = T.rowrank
        if not 0 < r < len(T.bonds):
            raise ValueError("rowrank must split the legs")
        self.T = T
        groups: Dict[tuple, List[int]] = {}
        for b, t in enumerate(T.itoi.tolist()):
            groups.setdefault(_row_charge(T, t), []).append(b)
        self.charges = sorted(groups)
        self.sectors = []
        for q in self.charges:
            bl = sorted(groups[q], key=lambda b: (tuple(T.itoi[b][:r]), tuple(T.itoi[b][r:])))
            rows = sorted({tuple(T.itoi[b][:r]) for b in bl})
            cols = sorted({tuple(T.itoi[b][r:]) for b in bl})
            rd = [int(np.prod([T.bonds[i].degs[x] for i, x in enumerate(rt)])) for rt in rows]
            cd = [int(np.prod([T.bonds[r + i].degs[x] for i, x in enumerate(ct)])) for ct in cols]
            ro, co = np.concatenate([[0], np.cumsum(rd)]), np.concatenate([[0], np.cumsum(cd)])
            M = np.zeros((ro[-1], co[-1]), dtype=T.dtype)
            for b in bl:
                i, j = rows.index(tuple(T.itoi[b][:r])), cols.index(tuple(T.itoi[b][r:]))
                M[ro[i]:ro[i + 1], co[j]:co[j + 1]] = T.blocks[b].reshape(rd[i], cd[j])
            U, s, Vh = np.linalg.svd(M, full_matrices=False)
            self.sectors.append({"rows": rows, "cols": cols, "ro": ro, "co": co, "U": U, "s": s, "Vh": Vh})

    def assemble(self, keep: Sequence[int]):
        """(S values per kept sector, U, vT) with sector i keeping its first keep[i] values."""
        T, r = self.T, self.T.rowrank
        kept = [i for i, k in enumerate(keep) if k > 0]
        syms = T.bonds[0].syms
        qn = np.array([self.charges[i] for i in kept], dtype=np.int64).reshape(len(kept), -1)
        degs = [int(keep[i]) for i in kept]
        aux_ket, aux_bra = Bond(-1, qn, degs, syms), Bond(1, qn, degs, syms)
        S = [self.sectors[i]["s"][:keep[i]].copy() for i in kept]
        u_bonds = list(T.bonds[:r]) + [aux_bra]
        u_blocks, u_itoi = [], []
        v_bonds = [aux_ket] + list(T.bonds[r:])
        v_blocks, v_itoi = [], []
        for new, i in enumerate(kept):
            sec, k = self.sectors[i], keep[i]
            for a, rt in enumerate(sec["rows"]):
                shp = [int(T.bonds[x].degs[y]) for x, y in enumerate(rt)] + [k]
                u_itoi.append(list(rt) + [new])
                u_blocks.append(sec["U"][sec["ro"][a]:sec["ro"][a + 1], :k].reshape(shp))
            for c, ct in enumerate(sec["cols"]):
                shp = [k] + [int(T.bonds[r + x].degs[y]) for x, y in enumerate(ct)]
                v_itoi.append([new] + list(ct))
                v_blocks.append(sec["Vh"][:k, sec["co"][c]:sec["co"][c + 1]].reshape(shp))
        U = _reorder(BlockTensor(u_bonds, list(T.labels[:r]) + ["_aux_L"], r, np.array(u_itoi, np.int64), u_blocks))
        vT = _reorder(BlockTensor(v_bonds, ["_aux_R"] + list(T.labels[r:]), 1, np.array(v_itoi, np.int64), v_blocks))
        return S, [self.charges[i] for i in kept], U, vT


def _reorder(t: BlockTensor) -> BlockTensor:
    """Blocks in BlockUniTensor::Init enumeration order of the tensor's bonds."""
    order = {tuple(x): i for i, x in enumerate(t.itoi.tolist())}
    itoi = enumerate_blocks(t.bonds)
    blocks = []
    for tup in itoi.tolist():
        i = order.get(tuple(tup))
        blocks.append(t.blocks[i] if i is not None else np.zeros(t.block_shape(tup), dtype=t.dtype))
    return BlockTensor(t.bonds, t.labels, t.rowrank, itoi, blocks)


def gesvd(T: BlockTensor):
    sv = BlockSvd(T)
    return sv.assemble([len(s["s"]) for s in sv.sectors])


def _cut(Sall: np.ndarray, keep_dim: int, err: float, floor: int):
    """Smin of the truncation rule on ascending values (Svd_truncate.cpp:166-191)."""
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


def svd_truncate(T: BlockTensor, keepdim: int, err: float = 0.0, mindim: int = 1):
    sv = BlockSvd(T)
    Sall = np.sort(np.concatenate([s["s"] for s in sv.sectors]))
    smin = _cut(Sall, int(keepdim), err, max(1, mindim))
    keep = [int(np.sum(s["s"] >= smin)) for s in sv.sectors]
    return sv.assemble(keep)


def gesvd_truncate(T: BlockTensor, keepdim: int, min_blockdim: Sequence[int], err: float = 0.0, mindim: int = 1):
    sv = BlockSvd(T)
    nb = len(sv.sectors)
    mb = list(min_blockdim) * nb if len(min_blockdim) == 1 else list(min_blockdim)
    if len(mb) != nb:
        raise ValueError("min_blockdim needs one entry per sector")
    keep_dim, min_dim = int(keepdim), max(1, mindim)
    rest, any_mb = [], False
    for b, s in enumerate(sv.sectors):
        v = s["s"]
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
    smin: Optional[float] = None
    if rest and keep_dim > 0:
        min_dim = max(1, min_dim) if not any_mb else max(0, min_dim)
        smin = _cut(np.sort(np.concatenate(rest)), keep_dim, err, min_dim)
    keep = []
    for b, s in enumerate(sv.sectors):
        v = s["s"]
        k = min(mb[b], len(v))
        if smin is not None:
            for i in range(len(v), mb[b], -1):
                if v[i - 1] >= smin:
                    k = i
                    break
        keep.append(k)
    return sv.assemble(keep)


def recompose(U: BlockTensor, S: List[np.ndarray], vT: BlockTensor, charges) -> BlockTensor:
    """U . diag(S) . vT back on the input's legs (blocks in the input's Init order)."""
    r = U.rowrank
    Ud = U.dense()
    Vd = vT.dense()
    s = np.concatenate(S)
    M = np.tensordot(Ud * s, Vd, axes=([r], [0]))
    bonds = list(U.bonds[:r]) + list(vT.bonds[1:])
    labels = list(U.labels[:r]) + list(vT.labels[1:])
    itoi = enumerate_blocks(bonds)
    offs = [np.concatenate([[0], np.cumsum(b.degs)[:-1]]) for b in bonds]
    blocks = []
    for t in itoi.tolist():
        sl = tuple(slice(offs[i][q], offs[i][q] + bonds[i].degs[q]) for i, q in enumerate(t))
        blocks.append(M[sl].copy())
    return BlockTensor(bonds, labels, r, itoi, blocks)
