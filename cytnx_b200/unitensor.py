"""UniTensor (dense and U(1)/Zn block-sparse) and Contract.

Mirrors ``cytnx::UniTensor`` (include/UniTensor.hpp) for the tensor-network hot path:
labels, bonds, rowrank, lazy ``permute`` (src/BlockUniTensor.cpp:588-708),
``contiguous``, ``relabel``, block access, ``Norm``, ``Dagger``/``Transpose``
(:1237-1245), arithmetic, and ``contract`` (:777-1235) / ``Contract``
(src/UniTensor_base.cpp:706-714).

Storage layout (B200): all blocks of a BlockUniTensor live in ONE flat device buffer,
back to back in the order BlockUniTensor::Init enumerates them (src/BlockUniTensor.cpp:
190-230).  A lazy permutation is one mapper shared by every block (the reference keeps
one per block; they are always equal).  ``contiguous()`` materialises all blocks with
the permute kernel; ``contract`` runs a cached plan: host-side block pairing once, then
one grouped-GEMM launch per call (cytnx_b200/csrc/blocks.cpp, gemm_f64.cu).
"""
from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from ._lib import BlockDesc, CytnxError
from .core import (Bond, Device, Symmetry, Tensor, Type, enumerate_blocks, require_cuda, BD_KET, BD_BRA,
                   BD_REG)


class UTenType:
    Void = -99
    Dense = 0
    Sparse = 1
    Block = 2


# ---------------------------------------------------------------- layouts
class BlockLayout:
    """Blocks of a tensor with given bonds, in enumeration order, packed back to back."""

    __slots__ = ("itoi", "shapes", "offs", "sizes", "nelem", "_index", "__weakref__")

    def __init__(self, bonds: Sequence[Bond], itoi: Optional[np.ndarray] = None):
        self.itoi = enumerate_blocks(bonds) if itoi is None else np.ascontiguousarray(itoi, dtype=np.int64)
        rank = len(bonds)
        degs = [b._degs for b in bonds]
        if rank:
            self.shapes = np.stack([degs[i][self.itoi[:, i]] for i in range(rank)], axis=1).astype(np.int64) \
                if len(self.itoi) else np.zeros((0, rank), dtype=np.int64)
        else:
            self.shapes = np.zeros((1, 0), dtype=np.int64)
        self.sizes = self.shapes.prod(axis=1).astype(np.int64) if len(self.shapes) else np.zeros(0, np.int64)
        self.offs = np.concatenate([[0], np.cumsum(self.sizes)[:-1]]).astype(np.int64) if len(self.sizes) else np.zeros(0, np.int64)
        self.nelem = int(self.sizes.sum())
        self._index = None

    def index(self) -> Dict[Tuple[int, ...], int]:
        if self._index is None:
            self._index = {tuple(t): i for i, t in enumerate(self.itoi.tolist())}
        return self._index


_LAYOUTS: Dict[tuple, BlockLayout] = {}


def layout_for(bonds: Sequence[Bond]) -> BlockLayout:
    key = tuple(b._sig() for b in bonds)
    lay = _LAYOUTS.get(key)
    if lay is None:
        lay = BlockLayout(bonds)
        _LAYOUTS[key] = lay
    return lay


class _LRU(dict):
    """Plan cache bounded to `cap` entries (least recently inserted evicted first)."""

    def __init__(self, cap: int):
        super().__init__()
        self.cap = cap

    def __setitem__(self, k, v):
        if k not in self and len(self) >= self.cap:
            del self[next(iter(self))]
        super().__setitem__(k, v)


_PLANS: Dict[tuple, object] = _LRU(512)


class _ContractPlan:
    def __init__(self, handle, keep):
        self.h = handle
        self.keep = keep  # layouts and arrays the plan was built from
        self.scratch = int(_lib.lib().ctn_contract_plan_scratch_bytes(handle))
        self.flops = float(_lib.lib().ctn_contract_plan_flops(handle))

    def __del__(self):
        try:
            _lib.lib().ctn_contract_plan_destroy(self.h)
        except Exception:
            pass


def _desc(lay: BlockLayout, mapper: Optional[Sequence[int]], itoi_logical: np.ndarray,
          shapes_logical: np.ndarray, keep: list) -> BlockDesc:
    rank = itoi_logical.shape[1] if itoi_logical.ndim == 2 else 0
    it = np.ascontiguousarray(itoi_logical, dtype=np.int64)
    sh = np.ascontiguousarray(shapes_logical, dtype=np.int64)
    of = np.ascontiguousarray(lay.offs, dtype=np.int64)
    keep += [it, sh, of]
    perm_ptr = None
    if mapper is not None and any(m != i for i, m in enumerate(mapper)):
        pm = np.ascontiguousarray(mapper, dtype=np.int64)
        keep.append(pm)
        perm_ptr = pm.ctypes.data
    return BlockDesc(rank, len(it), it.ctypes.data, sh.ctypes.data, of.ctypes.data, perm_ptr)


# ---------------------------------------------------------------- UniTensor
class UniTensor:
    """Labelled tensor with bonds; dense (one block) or block-sparse by quantum numbers."""

    def __init__(self, *args, labels: Sequence[str] = (), rowrank: int = -1, dtype: int = Type.Double,
                 device: Optional[int] = None, is_diag: bool = False, name: str = "", **kw):
        # UniTensor(bonds, labels=[], rowrank=-1, dtype, device, is_diag, name)
        # UniTensor(Tensor, is_diag=False, rowrank=-1, labels=[], name="")
        self._name = name
        self._is_diag = bool(is_diag)
        dev = Device.default if device is None else device
        if args and isinstance(args[0], Tensor):
            t = args[0]
            if len(args) > 1:
                self._is_diag = bool(args[1])
            if len(args) > 2:
                rowrank = args[2]
            if len(args) > 3:
                labels = args[3]
            self._kind = UTenType.Dense
            self._block = t
            self._bonds = [Bond(int(s)) for s in t.shape()]
            if self._is_diag:
                self._bonds = [Bond(int(t.shape()[0])), Bond(int(t.shape()[0]))]
            r = len(self._bonds)
            self._labels = [str(l) for l in labels] if labels else [str(i) for i in range(r)]
            self._rowrank = (1 if self._is_diag else (r // 2 if r else 0)) if rowrank < 0 else int(rowrank)
            self._is_braket = False
            return
        bonds = list(args[0]) if args else []
        if len(args) > 1:
            labels = args[1]
        if len(args) > 2:
            rowrank = args[2]
        if len(args) > 3:
            dtype = args[3]
        if len(args) > 4:
            dev = args[4]
        self._bonds = [b.clone() for b in bonds]
        r = len(bonds)
        labels = [str(l) for l in labels] if labels else [str(i) for i in range(r)]
        if len(labels) != r:
            raise CytnxError("[ERROR] labels must have same length as # of bonds.")
        if len(set(labels)) != len(labels):
            raise CytnxError("[ERROR] labels cannot contain duplicated elements.")
        self._labels = labels
        sym = r > 0 and all(b.has_symmetry() for b in bonds)
        if sym:
            self._kind = UTenType.Block
            nket = sum(1 for b in bonds if b.type() == BD_KET)
            self._rowrank = nket if rowrank < 0 else int(rowrank)
            if not (0 <= self._rowrank <= r):
                raise CytnxError("[ERROR][BlockUniTensor] rowrank must be >=0 and <=rank.")
            for b in bonds:
                if b.Nsym() != bonds[0].Nsym() or b.syms() != bonds[0].syms():
                    raise CytnxError("[ERROR][BlockUniTensor] symmetry mismatch between bonds")
            self._layout = layout_for(self._bonds)
            self._mapper = list(range(r))
            self._data = torch.zeros(self._layout.nelem, dtype=Type.to_torch(dtype), device=Device.torch_device(dev))
            self._is_braket = self._update_braket()
        else:
            if any(b.has_symmetry() for b in bonds):
                raise CytnxError("[ERROR] cannot mix symmetric and regular bonds")
            self._kind = UTenType.Dense
            shape = [b.dim() for b in bonds] if not self._is_diag else [bonds[0].dim()]
            self._block = Tensor(shape, dtype, dev)
            self._rowrank = (1 if self._is_diag else r // 2) if rowrank < 0 else int(rowrank)
            self._is_braket = False

    # -------------------------------------------------------------- internal constructors
    @classmethod
    def _new_block(cls, bonds, labels, rowrank, layout, mapper, data, name="") -> "UniTensor":
        u = cls.__new__(cls)
        u._name = name
        u._is_diag = False
        u._kind = UTenType.Block
        u._bonds = list(bonds)
        u._labels = list(labels)
        u._rowrank = int(rowrank)
        u._layout = layout
        u._mapper = list(mapper)
        u._data = data
        u._is_braket = u._update_braket()
        return u

    @classmethod
    def _new_dense(cls, block: Tensor, bonds, labels, rowrank, name="", is_diag=False) -> "UniTensor":
        u = cls.__new__(cls)
        u._name = name
        u._is_diag = is_diag
        u._kind = UTenType.Dense
        u._block = block
        u._bonds = list(bonds)
        u._labels = list(labels)
        u._rowrank = int(rowrank)
        u._is_braket = False
        return u

    def _update_braket(self) -> bool:
        if self._kind != UTenType.Block:
            return False
        return all(b.type() == BD_KET for b in self._bonds[: self._rowrank]) and \
            all(b.type() == BD_BRA for b in self._bonds[self._rowrank:])

    # -------------------------------------------------------------- metadata
    def uten_type(self) -> int:
        return self._kind

    def uten_type_str(self) -> str:
        return {UTenType.Dense: "Dense", UTenType.Block: "Block"}[self._kind]

    def is_blockform(self) -> bool:
        return self._kind == UTenType.Block

    def labels(self) -> List[str]:
        return list(self._labels)

    def bonds(self) -> List[Bond]:
        return list(self._bonds)

    def bond(self, idx) -> Bond:
        if isinstance(idx, str):
            idx = self._labels.index(idx)
        return self._bonds[idx]

    def rank(self) -> int:
        return len(self._bonds)

    def rowrank(self) -> int:
        return self._rowrank

    def shape(self) -> List[int]:
        return [b.dim() for b in self._bonds]

    def dtype(self) -> int:
        return Type.from_torch(self._storage_tensor().dtype)

    def dtype_str(self) -> str:
        return Type.getname(self.dtype())

    def device(self) -> int:
        return Device.from_torch(self._storage_tensor().device)

    def name(self) -> str:
        return self._name

    def is_diag(self) -> bool:
        return self._is_diag

    def is_braket_form(self) -> bool:
        return self._is_braket

    def is_contiguous(self) -> bool:
        if self._kind == UTenType.Block:
            return all(m == i for i, m in enumerate(self._mapper))
        return self._block.is_contiguous()

    def syms(self) -> List[Symmetry]:
        return self._bonds[0].syms() if self._bonds else []

    def Nblocks(self) -> int:
        return len(self._layout.itoi) if self._kind == UTenType.Block else 1

    def _storage_tensor(self) -> torch.Tensor:
        return self._data if self._kind == UTenType.Block else self._block._storage

    def set_name(self, name: str) -> "UniTensor":
        u = self.clone_meta()
        u._name = name
        return u

    def set_name_(self, name: str) -> "UniTensor":
        self._name = name
        return self

    def set_rowrank_(self, rowrank: int) -> "UniTensor":
        if not (0 <= rowrank <= self.rank()):
            raise CytnxError("[ERROR] rowrank out of range")
        self._rowrank = int(rowrank)
        self._is_braket = self._update_braket()
        return self

    def set_rowrank(self, rowrank: int) -> "UniTensor":
        return self.clone_meta().set_rowrank_(rowrank)

    def set_labels(self, labels: Sequence[str]) -> "UniTensor":
        labels = [str(l) for l in labels]
        if len(labels) != self.rank() or len(set(labels)) != len(labels):
            raise CytnxError("[ERROR] labels must be unique and match the rank")
        self._labels = labels
        return self

    def relabel_(self, *args) -> "UniTensor":
        if len(args) == 1:
            return self.set_labels(args[0])
        old, new = args
        if isinstance(old, (str, int)):
            old, new = [old], [new]
        labels = list(self._labels)
        for o, n in zip(old, new):
            labels[labels.index(str(o))] = str(n)
        return self.set_labels(labels)

    def relabel(self, *args) -> "UniTensor":
        return self.clone_meta().relabel_(*args)

    relabels_ = relabel_
    relabels = relabel

    def clone_meta(self) -> "UniTensor":
        if self._kind == UTenType.Block:
            return UniTensor._new_block(self._bonds, self._labels, self._rowrank, self._layout, self._mapper,
                                        self._data, self._name)
        return UniTensor._new_dense(self._block, self._bonds, self._labels, self._rowrank, self._name,
                                    self._is_diag)

    # -------------------------------------------------------------- block geometry
    def _logical_itoi(self) -> np.ndarray:
        return self._layout.itoi[:, self._mapper] if self.rank() else self._layout.itoi

    def _logical_shapes(self) -> np.ndarray:
        return self._layout.shapes[:, self._mapper] if self.rank() else self._layout.shapes

    def get_qindices(self, bidx: int) -> List[int]:
        return self._logical_itoi()[bidx].tolist()

    # -------------------------------------------------------------- permute / contiguous
    def _mapper_of(self, mapper) -> List[int]:
        if mapper and isinstance(mapper[0], str):
            idx = []
            for l in mapper:
                if l not in self._labels:
                    raise CytnxError(f"[ERROR][permute] Label '{l}' does not exist in UniTensor '{self._name}'.")
                idx.append(self._labels.index(l))
            mapper = idx
        mapper = [int(m) for m in mapper]
        if sorted(mapper) != list(range(self.rank())):
            raise CytnxError("[ERROR] invalid permutation")
        return mapper

    def permute(self, mapper, rowrank: int = -1) -> "UniTensor":
        """Metadata-only permutation of bonds, labels, qindices and (lazily) blocks."""
        m = self._mapper_of(list(mapper))
        if self._kind == UTenType.Block:
            u = UniTensor._new_block([self._bonds[i] for i in m], [self._labels[i] for i in m],
                                     self._rowrank if rowrank < 0 else rowrank, self._layout,
                                     [self._mapper[i] for i in m], self._data, self._name)
            if rowrank > self.rank():
                raise CytnxError("[ERROR][BlockUniTensor] rowrank cannot exceed the rank of UniTensor.")
            return u
        blk = self._block.permute(m) if not self._is_diag else self._block
        return UniTensor._new_dense(blk, [self._bonds[i] for i in m], [self._labels[i] for i in m],
                                    self._rowrank if rowrank < 0 else rowrank, self._name, self._is_diag)

    def permute_(self, mapper, rowrank: int = -1) -> "UniTensor":
        u = self.permute(mapper, rowrank)
        self.__dict__.update(u.__dict__)
        return self

    def contiguous(self) -> "UniTensor":
        if self.is_contiguous():
            return self
        if self._kind == UTenType.Dense:
            return UniTensor._new_dense(self._block.contiguous(), self._bonds, self._labels, self._rowrank,
                                        self._name, self._is_diag)
        require_cuda(self._data, "UniTensor::contiguous")
        lay_new = layout_for(self._bonds)
        # the logical enumeration order of the permuted bonds differs from the stored
        # order: materialise every block (permute kernel), then place blocks in the
        # new Init order.
        out = torch.empty(lay_new.nelem, dtype=self._data.dtype, device=self._data.device)
        itoi_l = self._logical_itoi()
        idx_new = lay_new.index()
        dst_offs = np.array([lay_new.offs[idx_new[tuple(t)]] for t in itoi_l.tolist()], dtype=np.int64)
        old_shapes = np.ascontiguousarray(self._layout.shapes, dtype=np.uint64)
        mp = np.ascontiguousarray(self._mapper, dtype=np.uint64)
        _lib.check(_lib.lib().ctn_permute_blocks(
            self._data.data_ptr(), out.data_ptr(), self.dtype(), self.rank(), len(itoi_l),
            old_shapes.ctypes.data_as(_lib.P_u64), self._layout.offs.ctypes.data_as(_lib.P_i64),
            dst_offs.ctypes.data_as(_lib.P_i64), mp.ctypes.data_as(_lib.P_u64), _lib.stream_ptr()),
            "BlockUniTensor::contiguous")
        return UniTensor._new_block(self._bonds, self._labels, self._rowrank, lay_new, list(range(self.rank())),
                                    out, self._name)

    def contiguous_(self) -> "UniTensor":
        u = self.contiguous()
        self.__dict__.update(u.__dict__)
        return self

    # -------------------------------------------------------------- blocks
    def get_block_(self, idx: Union[int, Sequence[int]] = 0) -> Tensor:
        if self._kind == UTenType.Dense:
            return self._block
        if not isinstance(idx, (int, np.integer)):
            key = tuple(int(i) for i in idx)
            hits = [b for b, t in enumerate(self._logical_itoi().tolist()) if tuple(t) == key]
            if not hits:
                raise CytnxError("[ERROR] no block with the given qnum indices")
            idx = hits[0]
        idx = int(idx)
        off, sz = int(self._layout.offs[idx]), int(self._layout.sizes[idx])
        t = Tensor.__new__(Tensor)
        t._storage = self._data[off: off + sz]
        phys = self._layout.shapes[idx].tolist()
        t._shape = phys
        t._mapper = list(range(len(phys)))
        t._invmapper = list(range(len(phys)))
        t._contiguous = True
        return t.permute(self._mapper) if self.rank() else t

    def get_block(self, idx=0) -> Tensor:
        return self.get_block_(idx).clone()

    def get_blocks_(self) -> List[Tensor]:
        if self._kind == UTenType.Dense:
            return [self._block]
        return [self.get_block_(i) for i in range(self.Nblocks())]

    def get_blocks(self) -> List[Tensor]:
        return [b.clone() for b in self.get_blocks_()]

    def put_block_(self, t: Tensor, idx: Union[int, Sequence[int]] = 0) -> "UniTensor":
        return self.put_block(t, idx)

    def put_block(self, t: Tensor, idx: Union[int, Sequence[int]] = 0) -> "UniTensor":
        if self._kind == UTenType.Dense:
            if t.shape() != self._block.shape():
                raise CytnxError("[ERROR] put_block: shape mismatch")
            self._block = t.clone().to(self.device()) if t.device() != self.device() else t.clone()
            return self
        dst = self.get_block_(idx)
        if t.shape() != dst.shape():
            raise CytnxError("[ERROR] put_block: shape mismatch")
        if not self.is_contiguous():
            self.contiguous_()
            dst = self.get_block_(idx)
        src = t.to_torch() if t._storage.is_cuda else torch.from_numpy(t.numpy())
        dst._storage.copy_(src.reshape(-1).to(dst._storage.device, dst._storage.dtype))
        return self

    def _locate(self, locator: Sequence[int]):
        """Global element index -> (block index, index inside the block) (_fx_locate_elem)."""
        qidx, inner = [], []
        for i, g in enumerate(locator):
            degs = self._bonds[i]._degs
            acc = 0
            for q, d in enumerate(degs):
                if g < acc + d:
                    qidx.append(q)
                    inner.append(int(g - acc))
                    break
                acc += d
            else:
                raise CytnxError("[ERROR] locator out of range")
        key = tuple(qidx)
        for b, t in enumerate(self._logical_itoi().tolist()):
            if tuple(t) == key:
                return b, inner
        return -1, inner

    def at(self, locator: Sequence[int]):
        if self._kind == UTenType.Dense:
            a = self._block.numpy()
            return a[tuple(locator)]
        b, inner = self._locate(locator)
        if b < 0:
            return 0.0
        return self.get_block_(b).numpy()[tuple(inner)]

    def elem_exists(self, locator: Sequence[int]) -> bool:
        return self._kind == UTenType.Dense or self._locate(locator)[0] >= 0

    def set_elem(self, locator: Sequence[int], value) -> "UniTensor":
        if self._kind == UTenType.Dense:
            c = self._block.contiguous()
            shp = c.shape()
            flat = int(np.ravel_multi_index(tuple(locator), shp))
            c._storage[flat] = value
            self._block = c
            return self
        b, inner = self._locate(locator)
        if b < 0:
            raise CytnxError("[ERROR] set_elem: the element is not in any symmetry-allowed block")
        self.contiguous_()
        shp = self._layout.shapes[b].tolist()
        flat = int(self._layout.offs[b]) + int(np.ravel_multi_index(tuple(inner), shp))
        self._data[flat] = value
        return self

    # -------------------------------------------------------------- conversion
    def to_dense_numpy(self) -> np.ndarray:
        """Every block placed at its sector offsets (a checking aid)."""
        if self._kind == UTenType.Dense:
            return self._block.numpy()
        offs = [np.concatenate([[0], np.cumsum(b._degs)[:-1]]) for b in self._bonds]
        npdt = torch.empty(0, dtype=self._data.dtype).numpy().dtype
        full = np.zeros(self.shape(), dtype=npdt)
        for b, t in enumerate(self._logical_itoi().tolist()):
            sl = tuple(slice(offs[i][q], offs[i][q] + self._bonds[i]._degs[q]) for i, q in enumerate(t))
            full[sl] = self.get_block_(b).numpy()
        return full

    def to(self, device: int) -> "UniTensor":
        u = self.clone_meta()
        if self._kind == UTenType.Block:
            u._data = self._data.to(Device.torch_device(device))
        else:
            u._block = self._block.to(device)
        return u

    def to_(self, device: int) -> "UniTensor":
        self.__dict__.update(self.to(device).__dict__)
        return self

    def clone(self) -> "UniTensor":
        u = self.clone_meta()
        if self._kind == UTenType.Block:
            u._data = self._data.clone()
        else:
            u._block = self._block.clone()
        return u

    def astype(self, dtype: int) -> "UniTensor":
        u = self.clone_meta()
        if self._kind == UTenType.Block:
            u._data = self._data.to(Type.to_torch(dtype))
        else:
            u._block = self._block.astype(dtype)
        return u

    def item(self):
        t = self._storage_tensor()
        if t.numel() != 1:
            raise CytnxError("[ERROR] item() requires exactly one element")
        return t.item()

    # -------------------------------------------------------------- flat data (Lanczos / autograd)
    def flat_view(self) -> torch.Tensor:
        """The contiguous block storage as one 1-D torch tensor (zero-copy)."""
        u = self.contiguous()
        return u._data if u._kind == UTenType.Block else u._block.to_torch().reshape(-1)

    def with_flat(self, flat: torch.Tensor) -> "UniTensor":
        """A tensor of the same (contiguous) structure viewing ``flat``."""
        u = self.contiguous().clone_meta()
        if u._kind == UTenType.Block:
            if flat.numel() != u._layout.nelem:
                raise CytnxError("[ERROR] flat buffer size mismatch")
            u._data = flat
        else:
            u._block = Tensor.from_torch(flat.reshape(u._block.shape()))
        return u

    # -------------------------------------------------------------- norms / arithmetic
    def Norm(self) -> Tensor:
        return Tensor.from_torch(torch.tensor([self.norm()], dtype=torch.float64))

    def norm(self) -> float:
        t = self._storage_tensor()
        if t.is_cuda and t.dtype == torch.float64 and t.numel() > 0:
            out = torch.empty(1, dtype=torch.float64, device=t.device)
            _lib.check(_lib.lib().ctn_nrm2_f64(t.data_ptr(), t.numel(), out.data_ptr(), _lib.stream_ptr()), "Norm")
            return float(out.item())
        require_cuda(t, "Norm")
        return float(torch.linalg.vector_norm(t).item())

    def normalize_(self) -> "UniTensor":
        n = self.norm()
        self._storage_tensor().div_(n)
        return self

    def _binary(self, other, op, inplace=False):
        if isinstance(other, UniTensor):
            a = self.contiguous()
            b = other.contiguous()
            if b._labels != a._labels:
                b = b.permute(a._labels).contiguous()
            if a._kind != b._kind or a.shape() != b.shape():
                raise CytnxError("[ERROR] arithmetic between UniTensors of different structure")
            if a._kind == UTenType.Block and not np.array_equal(a._layout.itoi, b._layout.itoi):
                raise CytnxError("[ERROR] arithmetic between BlockUniTensors with different blocks")
            x, y = a._storage_tensor(), b._storage_tensor()
        else:
            a = self.contiguous()
            x, y = a._storage_tensor(), other
        r = op(x, y)
        if inplace:
            self.__dict__.update(a.with_flat(r).__dict__)
            return self
        return a.with_flat(r)

    def __add__(self, o):
        return self._binary(o, lambda x, y: x + y)

    def __radd__(self, o):
        return self._binary(o, lambda x, y: y + x)

    def __sub__(self, o):
        return self._binary(o, lambda x, y: x - y)

    def __rsub__(self, o):
        return self._binary(o, lambda x, y: y - x)

    def __mul__(self, o):
        return self._binary(o, lambda x, y: x * y)

    def __rmul__(self, o):
        return self._binary(o, lambda x, y: y * x)

    def __truediv__(self, o):
        return self._binary(o, lambda x, y: x / y)

    def __iadd__(self, o):
        return self._binary(o, lambda x, y: x + y, True)

    def __isub__(self, o):
        return self._binary(o, lambda x, y: x - y, True)

    def __imul__(self, o):
        return self._binary(o, lambda x, y: x * y, True)

    def __itruediv__(self, o):
        return self._binary(o, lambda x, y: x / y, True)

    def __neg__(self):
        return self._binary(-1.0, lambda x, y: x * y)

    def Conj(self) -> "UniTensor":
        u = self.clone_meta()
        if self._kind == UTenType.Block:
            u._data = torch.conj(self._data).resolve_conj() if self._data.is_complex() else self._data
        else:
            u._block = Tensor.from_torch(torch.conj(self._block.to_torch()).resolve_conj()) \
                if self._block._storage.is_complex() else self._block
        return u

    def Transpose(self) -> "UniTensor":
        """BlockUniTensor::Transpose_ (src/BlockUniTensor.cpp:1237-1245): redirect every bond,
        reverse the leg order, rowrank -> rank - rowrank."""
        r = self.rank()
        u = self.clone_meta()
        if self._kind == UTenType.Block:
            u._bonds = [b.redirect() for b in self._bonds]
            # redirected bonds enumerate the same blocks: the stored layout stays valid
            u._layout = self._layout
        return u.permute(list(range(r - 1, -1, -1)), r - self._rowrank)

    def Transpose_(self) -> "UniTensor":
        self.__dict__.update(self.Transpose().__dict__)
        return self

    def Dagger(self) -> "UniTensor":
        return self.Conj().Transpose()

    def Dagger_(self) -> "UniTensor":
        self.__dict__.update(self.Dagger().__dict__)
        return self

    # -------------------------------------------------------------- contract
    def contract(self, rhs: "UniTensor") -> "UniTensor":
        return Contract(self, rhs)

    # -------------------------------------------------------------- save / load
    def Save(self, fname: str) -> None:
        from . import fileio

        if not fname.endswith(".cytnx"):
            fname = fname + ".cytnx"
        u = self.contiguous()
        bonds = [{"type": b.type(), "nsym": b.Nsym(), "qnums": b._qnums, "degs": b._degs, "dim": b.dim(),
                  "syms": [{"stype": s.stype, "n": s.n} for s in b.syms()]} for b in u._bonds]
        d = {"uten_type": u._kind, "is_braket_form": u._is_braket, "is_tag": u._kind == UTenType.Block,
             "is_diag": u._is_diag, "rowrank": u._rowrank, "name": u._name, "labels": u._labels,
             "bonds": bonds}
        if u._kind == UTenType.Block:
            d["itoi"] = u._layout.itoi
            d["blocks"] = [u.get_block_(i).numpy() for i in range(u.Nblocks())]
        else:
            d["block"] = u._block.numpy()
        fileio.write_unitensor(fname, d)

    @staticmethod
    def Load(fname: str, device: Optional[int] = None) -> "UniTensor":
        from . import fileio

        d = fileio.read_unitensor(fname)
        return UniTensor.from_parsed(d, device)

    @staticmethod
    def from_parsed(d, device: Optional[int] = None) -> "UniTensor":
        dev = Device.default if device is None else device
        bonds = []
        for b in d["bonds"]:
            if len(b["degs"]) and b["nsym"]:
                bonds.append(Bond(b["type"], b["qnums"], b["degs"], [Symmetry(s["stype"], s["n"]) for s in b["syms"]]))
            else:
                bonds.append(Bond(int(b["dim"]), b["type"]))
        if d["uten_type"] == UTenType.Block:
            u = UniTensor(bonds, labels=d["labels"], rowrank=d["rowrank"],
                          dtype=Type.from_torch(torch.from_numpy(d["blocks"][0][:0].copy()).dtype) if d["blocks"] else Type.Double,
                          device=dev, name=d.get("name", ""))
            idx = u._layout.index()
            for t, blk in zip(np.asarray(d["itoi"]).tolist(), d["blocks"]):
                b = idx[tuple(t)]
                off = int(u._layout.offs[b])
                u._data[off: off + blk.size] = torch.from_numpy(np.ascontiguousarray(blk).reshape(-1)).to(u._data.device)
            return u
        t = Tensor.from_numpy(d["block"], dev)
        return UniTensor(t, d["is_diag"], d["rowrank"], d["labels"], name=d.get("name", ""))

    def __repr__(self):
        return (f"UniTensor(name='{self._name}', type={self.uten_type_str()}, labels={self._labels}, "
                f"shape={self.shape()}, rowrank={self._rowrank}, blocks={self.Nblocks()})")

    def print_diagram(self):
        print(repr(self))
        for l, b in zip(self._labels, self._bonds):
            print(f"  {l}: {b}")


# ---------------------------------------------------------------- Contract
def _dense_as_block_desc(u: UniTensor, keep: list):
    t = u._block
    shape = t.shape()
    it = np.zeros((1, len(shape)), dtype=np.int64)
    sh = np.asarray([shape], dtype=np.int64)
    of = np.zeros(1, dtype=np.int64)
    keep += [it, sh, of]
    perm_ptr = None
    if not t.is_contiguous():
        pm = np.ascontiguousarray(t._mapper, dtype=np.int64)
        keep.append(pm)
        perm_ptr = pm.ctypes.data
    return BlockDesc(len(shape), 1, it.ctypes.data, sh.ctypes.data, of.ctypes.data, perm_ptr)


def Contract(A: UniTensor, B: UniTensor, cacheL: bool = False, cacheR: bool = False) -> UniTensor:
    """Contract the common labels of A and B (src/UniTensor_base.cpp:706-714)."""
    if A._kind != B._kind:
        raise CytnxError("[ERROR][contract] Cannot contract BlockUniTensor with other type of UniTensor.")
    comm = sorted(set(A._labels) & set(B._labels))  # vec_intersect_: sorted common labels
    c1 = [A._labels.index(l) for l in comm]
    c2 = [B._labels.index(l) for l in comm]
    n1 = [i for i in range(A.rank()) if i not in c1]
    n2 = [i for i in range(B.rank()) if i not in c2]
    if A._kind == UTenType.Block:
        if A.syms() != B.syms():
            raise CytnxError("[ERROR][BlockUniTensor][contract] Two UniTensor have different symmetry types, cannot contract.")
        for l, i, j in zip(comm, c1, c2):
            if A._bonds[i].type() + B._bonds[j].type() != 0:
                raise CytnxError(f"[ERROR][BlockUniTensor][contract] A bond with type BRA can only be contracted with type KET. Invalid contraction for label '{l}'.")
            if not (np.array_equal(A._bonds[i]._qnums, B._bonds[j]._qnums) and np.array_equal(A._bonds[i]._degs, B._bonds[j]._degs)):
                raise CytnxError(f"[ERROR][BlockUniTensor][contract] Contracted bond with label '{l}' has a qnum/degeneracy mismatch.")
    else:
        for l, i, j in zip(comm, c1, c2):
            if A._bonds[i].dim() != B._bonds[j].dim():
                raise CytnxError(f"[ERROR][contract] dimension mismatch on label '{l}'")
    if not comm:
        return _outer(A, B)
    if not n1 and not n2:
        return _full_contract(A, B, c1, c2)
    out_bonds = [A._bonds[i].clone() for i in n1] + [B._bonds[i].clone() for i in n2]
    out_labels = [A._labels[i] for i in n1] + [B._labels[i] for i in n2]
    out_rowrank = A._rowrank + B._rowrank - sum(1 for i in c1 if i < A._rowrank) - sum(1 for i in c2 if i < B._rowrank)
    dtA, dtB = A._storage_tensor().dtype, B._storage_tensor().dtype
    if dtA != torch.float64 or dtB != torch.float64:
        raise CytnxError("[ERROR][contract] the device contraction engine computes in float64 "
                         f"(got {dtA} x {dtB}); convert with astype(Type.Double)")
    require_cuda(A._storage_tensor(), "contract")
    require_cuda(B._storage_tensor(), "contract")
    keep: list = []
    if A._kind == UTenType.Block:
        lay_out = layout_for(out_bonds)
        key = (id(A._layout), tuple(A._mapper), id(B._layout), tuple(B._mapper), tuple(c1), tuple(c2), id(lay_out))
        plan = _PLANS.get(key)
        if plan is None:
            dA = _desc(A._layout, A._mapper, A._logical_itoi(), A._logical_shapes(), keep)
            dB = _desc(B._layout, B._mapper, B._logical_itoi(), B._logical_shapes(), keep)
            dO = _desc(lay_out, None, lay_out.itoi, lay_out.shapes, keep)
            plan = _make_plan(dA, dB, c1, c2, dO, keep + [A._layout, B._layout, lay_out])
            _PLANS[key] = plan
        out = torch.empty(lay_out.nelem, dtype=torch.float64, device=A._data.device)
        _run_plan(plan, A._data, B._data, out)
        return UniTensor._new_block(out_bonds, out_labels, out_rowrank, lay_out, list(range(len(out_bonds))), out)
    # dense: one block each
    shapeA, shapeB = A._block.shape(), B._block.shape()
    key = ("dense", tuple(shapeA), tuple(A._block._mapper), tuple(shapeB), tuple(B._block._mapper), tuple(c1), tuple(c2))
    out_shape = [shapeA[i] for i in n1] + [shapeB[i] for i in n2]
    plan = _PLANS.get(key)
    if plan is None:
        dA = _dense_as_block_desc(A, keep)
        dB = _dense_as_block_desc(B, keep)
        it = np.zeros((1, len(out_shape)), dtype=np.int64)
        sh = np.asarray([out_shape], dtype=np.int64)
        of = np.zeros(1, dtype=np.int64)
        keep += [it, sh, of]
        dO = BlockDesc(len(out_shape), 1, it.ctypes.data, sh.ctypes.data, of.ctypes.data, None)
        plan = _make_plan(dA, dB, c1, c2, dO, keep)
        _PLANS[key] = plan
    out = torch.empty(int(np.prod(out_shape)), dtype=torch.float64, device=A._block._storage.device)
    _run_plan(plan, A._block._storage, B._block._storage, out)
    blk = Tensor.from_torch(out.view(*out_shape))
    return UniTensor._new_dense(blk, out_bonds, out_labels, out_rowrank)


def _make_plan(dA, dB, c1, c2, dO, keep) -> _ContractPlan:
    h = ctypes.c_void_p()
    c1a = np.ascontiguousarray(c1, dtype=np.int64)
    c2a = np.ascontiguousarray(c2, dtype=np.int64)
    _lib.check(_lib.lib().ctn_contract_plan_create(ctypes.byref(dA), ctypes.byref(dB), len(c1),
                                                   c1a.ctypes.data_as(_lib.P_i64), c2a.ctypes.data_as(_lib.P_i64),
                                                   ctypes.byref(dO), ctypes.byref(h)), "BlockUniTensor::contract")
    return _ContractPlan(h.value, keep)


def _run_plan(plan: _ContractPlan, a: torch.Tensor, b: torch.Tensor, out: torch.Tensor) -> None:
    scratch = torch.empty(max(plan.scratch, 16), dtype=torch.uint8, device=a.device)
    _lib.check(_lib.lib().ctn_contract_execute(plan.h, 3, a.data_ptr(), b.data_ptr(), out.data_ptr(),
                                               scratch.data_ptr(), _lib.stream_ptr()), "contract")


def contract_plan_flops(A: UniTensor, B: UniTensor) -> float:
    """2*m*n*k over all block pairs that BlockUniTensor::contract(A, B) multiplies (host only)."""
    comm = sorted(set(A._labels) & set(B._labels))
    c1 = [A._labels.index(l) for l in comm]
    c2 = [B._labels.index(l) for l in comm]
    n1 = [i for i in range(A.rank()) if i not in c1]
    n2 = [i for i in range(B.rank()) if i not in c2]
    out_bonds = [A._bonds[i] for i in n1] + [B._bonds[i] for i in n2]
    keep: list = []
    lay_out = layout_for(out_bonds)
    dA = _desc(A._layout, A._mapper, A._logical_itoi(), A._logical_shapes(), keep)
    dB = _desc(B._layout, B._mapper, B._logical_itoi(), B._logical_shapes(), keep)
    dO = _desc(lay_out, None, lay_out.itoi, lay_out.shapes, keep)
    plan = _make_plan(dA, dB, c1, c2, dO, keep)
    return plan.flops


def structure_only(bonds: Sequence[Bond], labels: Sequence[str], rowrank: int = -1) -> UniTensor:
    """A BlockUniTensor skeleton with no storage (for host-side planning and counting)."""
    u = UniTensor.__new__(UniTensor)
    u._name = ""
    u._is_diag = False
    u._kind = UTenType.Block
    u._bonds = [b.clone() for b in bonds]
    u._labels = [str(l) for l in labels]
    u._rowrank = sum(1 for b in bonds if b.type() == BD_KET) if rowrank < 0 else rowrank
    u._layout = layout_for(u._bonds)
    u._mapper = list(range(len(bonds)))
    u._data = torch.empty(0, dtype=torch.float64)
    u._is_braket = u._update_braket()
    return u


def _full_contract(A: UniTensor, B: UniTensor, c1, c2) -> UniTensor:
    """All legs contracted: sum over matching blocks of a dot product (:886-946)."""
    Ap = A.permute(c1).contiguous()
    Bp = B.permute(c2).contiguous()
    if A._kind == UTenType.Block:
        require_cuda(Ap._data, "contract")
        ia, ib = Ap._layout.index(), Bp._layout.index()
        s = torch.zeros((), dtype=torch.promote_types(Ap._data.dtype, Bp._data.dtype), device=Ap._data.device)
        if np.array_equal(Ap._layout.itoi, Bp._layout.itoi):
            s = torch.dot(Ap._data, Bp._data.to(Ap._data.dtype))
        else:
            for t, a in ia.items():
                b = ib.get(t)
                if b is None:
                    continue
                oa, sa = int(Ap._layout.offs[a]), int(Ap._layout.sizes[a])
                ob = int(Bp._layout.offs[b])
                s = s + torch.dot(Ap._data[oa: oa + sa], Bp._data[ob: ob + sa])
        blk = Tensor.from_torch(s.reshape(()))
    else:
        x = Ap._block.to_torch().reshape(-1)
        y = Bp._block.to_torch().reshape(-1)
        blk = Tensor.from_torch(torch.dot(x, y.to(x.dtype)).reshape(()))
    return UniTensor._new_dense(blk, [], [], 0)


def _outer(A: UniTensor, B: UniTensor) -> UniTensor:
    """No common label: Kronecker product of blocks (BlockUniTensor.cpp:801-862)."""
    out_bonds = [b.clone() for b in A._bonds] + [b.clone() for b in B._bonds]
    out_labels = A._labels + B._labels
    rr = A._rowrank + B._rowrank
    if A._kind == UTenType.Dense:
        x, y = A._block.to_torch(), B._block.to_torch()
        blk = Tensor.from_torch(torch.tensordot(x, y, dims=0))
        return UniTensor._new_dense(blk, out_bonds, out_labels, rr)
    Ac, Bc = A.contiguous(), B.contiguous()
    out = UniTensor(out_bonds, labels=out_labels, rowrank=rr, dtype=A.dtype(), device=A.device())
    ia, ib = Ac._layout.index(), Bc._layout.index()
    ra = A.rank()
    for t, ob in out._layout.index().items():
        a, b = ia.get(t[:ra]), ib.get(t[ra:])
        if a is None or b is None:
            continue
        x = Ac.get_block_(a).to_torch()
        y = Bc.get_block_(b).to_torch()
        off, sz = int(out._layout.offs[ob]), int(out._layout.sizes[ob])
        out._data[off: off + sz] = torch.tensordot(x, y, dims=0).reshape(-1)
    return out
