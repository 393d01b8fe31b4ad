"""Type/Device constants, Symmetry, Bond and the dense Tensor (lazy permute).

Mirrors the reference's ``cytnx::Type`` ids (include/Type.hpp:177-179), ``Symmetry``
(src/Symmetry.cpp), ``Bond`` (include/Bond.hpp:31-71) and ``Tensor`` with its lazy
``permute`` / ``contiguous`` semantics (src/backend/Tensor_impl.cpp:38-143,
include/backend/Tensor_impl.hpp:222-325).  Storage is a 1-D torch tensor; every
data movement on a CUDA tensor runs the library's own kernels through the C ABI.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import CytnxError


class _Type:
    Void = 0
    ComplexDouble = 1
    ComplexFloat = 2
    Double = 3
    Float = 4
    Int64 = 5
    Uint64 = 6
    Int32 = 7
    Uint32 = 8
    Int16 = 9
    Uint16 = 10
    Bool = 11

    _torch = {1: torch.complex128, 2: torch.complex64, 3: torch.float64, 4: torch.float32,
              5: torch.int64, 6: torch.uint64, 7: torch.int32, 8: torch.uint32, 9: torch.int16,
              10: torch.uint16, 11: torch.bool}
    _names = {1: "Complex Double (Complex Float64)", 2: "Complex Float (Complex Float32)",
              3: "Double (Float64)", 4: "Float (Float32)", 5: "Int64", 6: "Uint64", 7: "Int32",
              8: "Uint32", 9: "Int16", 10: "Uint16", 11: "Bool"}

    def to_torch(self, dt: int) -> torch.dtype:
        return self._torch[dt]

    def from_torch(self, dt: torch.dtype) -> int:
        for k, v in self._torch.items():
            if v == dt:
                return k
        raise CytnxError(f"unsupported dtype {dt}")

    def getname(self, dt: int) -> str:
        return self._names.get(dt, "Void")

    def is_float(self, dt: int) -> bool:
        return dt in (1, 2, 3, 4)

    def is_complex(self, dt: int) -> bool:
        return dt in (1, 2)


Type = _Type()


class _Device:
    cpu = -1
    cuda = 0

    @property
    def Ngpus(self) -> int:
        return torch.cuda.device_count()

    @property
    def default(self) -> int:
        return 0 if torch.cuda.is_available() else -1

    def torch_device(self, dev: int) -> torch.device:
        return torch.device("cpu") if dev < 0 else torch.device(f"cuda:{dev}")

    def from_torch(self, d: torch.device) -> int:
        return -1 if d.type == "cpu" else (d.index or 0)


Device = _Device()


def require_cuda(t: torch.Tensor, what: str) -> None:
    if t.device.type != "cuda":
        raise CytnxError(f"[{what}] cytnx_b200 computes on CUDA devices only; "
                         f"move the tensor to a GPU with .to(cytnx_b200.Device.cuda)")


# ---------------------------------------------------------------- Symmetry
class Symmetry:
    """U1 (stype -1) or Zn (stype 0, modulus n) -- src/Symmetry.cpp:33-108."""

    def __init__(self, stype: int = -1, n: int = 1):
        self.stype, self.n = int(stype), int(n)

    @staticmethod
    def U1() -> "Symmetry":
        return Symmetry(-1, 1)

    @staticmethod
    def Zn(n: int) -> "Symmetry":
        return Symmetry(0, n)

    def combine_rule(self, a: int, b: int) -> int:
        return (a + b) % self.n if self.stype == 0 else a + b

    def reverse_rule(self, a: int) -> int:
        return (self.n - a) % self.n if self.stype == 0 else -a

    def stype_str(self) -> str:
        return "U1" if self.stype == -1 else f"Z{self.n}"

    def __eq__(self, o) -> bool:
        return isinstance(o, Symmetry) and (self.stype, self.n) == (o.stype, o.n)

    def __hash__(self):
        return hash((self.stype, self.n))

    def __repr__(self):
        return f"Symmetry({self.stype_str()})"


# ---------------------------------------------------------------- Bond
BD_KET, BD_BRA, BD_REG, BD_NONE, BD_IN, BD_OUT = -1, 1, 0, 0, -1, 1


class _BondType:
    BD_KET, BD_BRA, BD_REG, BD_NONE, BD_IN, BD_OUT = -1, 1, 0, 0, -1, 1


bondType = _BondType()


class Bond:
    """A leg: type (ket -1 / bra +1 / regular 0), qnums [nq][nsym], degeneracies, symmetries."""

    def __init__(self, *args, **kw):
        # Bond(dim) | Bond(dim, type) | Bond(type, qnums, degs, syms=None)
        if args and isinstance(args[0], (int, np.integer)) and (len(args) == 1 or (len(args) == 2 and not isinstance(args[1], (list, tuple)))):
            self._dim = int(args[0])
            self._type = int(args[1]) if len(args) > 1 else int(kw.get("bd_type", BD_REG))
            self._qnums = np.zeros((0, 0), dtype=np.int64)
            self._degs = np.zeros(0, dtype=np.int64)
            self._syms: List[Symmetry] = []
            return
        btype, qnums, degs = args[0], args[1], args[2]
        syms = args[3] if len(args) > 3 else kw.get("syms", None)
        self._type = int(btype)
        q = np.asarray(qnums, dtype=np.int64)
        if q.ndim == 1:
            q = q.reshape(-1, 1)
        self._qnums = q
        self._degs = np.asarray(degs, dtype=np.int64)
        if len(self._degs) != len(self._qnums):
            raise CytnxError("[Bond] qnums and degs must have the same length")
        if syms is None:
            syms = [Symmetry.U1() for _ in range(q.shape[1])]
        self._syms = list(syms)
        for s, col in zip(self._syms, q.T):
            if s.stype == 0 and ((col < 0) | (col >= s.n)).any():
                raise CytnxError(f"[Bond] qnum out of range for {s.stype_str()}")
        self._dim = int(self._degs.sum())

    # accessors (include/Bond.hpp)
    def dim(self) -> int:
        return self._dim

    def type(self) -> int:
        return self._type

    def qnums(self) -> List[List[int]]:
        return self._qnums.tolist()

    def getDegeneracies(self) -> List[int]:
        return self._degs.tolist()

    def syms(self) -> List[Symmetry]:
        return list(self._syms)

    def Nsym(self) -> int:
        return len(self._syms)

    def has_symmetry(self) -> bool:
        return len(self._degs) > 0

    def redirect(self) -> "Bond":
        b = self.clone()
        b._type = -self._type
        return b

    def clone(self) -> "Bond":
        b = Bond.__new__(Bond)
        b._dim, b._type = self._dim, self._type
        b._qnums, b._degs, b._syms = self._qnums.copy(), self._degs.copy(), list(self._syms)
        return b

    def __eq__(self, o) -> bool:
        return (isinstance(o, Bond) and self._type == o._type and self._dim == o._dim
                and np.array_equal(self._qnums, o._qnums) and np.array_equal(self._degs, o._degs)
                and self._syms == o._syms)

    def __repr__(self):
        t = {-1: "KET", 1: "BRA", 0: "REG"}[self._type]
        if not self.has_symmetry():
            return f"Bond(dim={self._dim}, {t})"
        return f"Bond({t}, qnums={self.qnums()}, degs={self.getDegeneracies()})"

    def _sig(self):
        return (self._type, self._dim, self._qnums.tobytes(), self._degs.tobytes(),
                tuple((s.stype, s.n) for s in self._syms))


def enumerate_blocks(bonds: Sequence[Bond]) -> np.ndarray:
    """BlockUniTensor::Init block enumeration through the C ABI (host code)."""
    rank = len(bonds)
    if rank == 0:
        return np.zeros((1, 0), dtype=np.int64)
    nsym = bonds[0].Nsym()
    st = np.array([s.stype for s in bonds[0].syms()], dtype=np.int32)
    sn = np.array([s.n for s in bonds[0].syms()], dtype=np.int64)
    bt = np.array([b.type() for b in bonds], dtype=np.int32)
    nqs = np.array([len(b._degs) for b in bonds], dtype=np.int64)
    tabs = [np.ascontiguousarray(b._qnums, dtype=np.int64) for b in bonds]
    ptrs = (ctypes.c_void_p * rank)(*[t.ctypes.data for t in tabs])
    cap = int(np.prod([max(1, int(n)) for n in nqs]))
    out = np.zeros((max(cap, 1), rank), dtype=np.int64)
    cnt = ctypes.c_int64(0)
    _lib.check(_lib.lib().ctn_blocks_enumerate(
        rank, nsym, st.ctypes.data_as(_lib.P_i32), sn.ctypes.data_as(_lib.P_i64),
        bt.ctypes.data_as(_lib.P_i32), nqs.ctypes.data_as(_lib.P_i64), ptrs,
        out.ctypes.data_as(_lib.P_i64), cap, ctypes.byref(cnt)), "BlockUniTensor::Init")
    return out[: cnt.value].copy()


# ---------------------------------------------------------------- Tensor
def _u64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


def device_permute(src: torch.Tensor, old_shape: Sequence[int], mapper: Sequence[int]) -> torch.Tensor:
    """out = src (row-major, old_shape) permuted by mapper, on the device (ctn_permute)."""
    require_cuda(src, "permute")
    n = int(np.prod(old_shape)) if len(old_shape) else 1
    out = torch.empty(n, dtype=src.dtype, device=src.device)
    if n == 0:
        return out
    dt = Type.from_torch(src.dtype)
    shp, mp = _u64(old_shape), _u64(mapper)
    _lib.check(_lib.lib().ctn_permute(src.data_ptr(), out.data_ptr(), dt, len(old_shape),
                                      shp.ctypes.data_as(_lib.P_u64), mp.ctypes.data_as(_lib.P_u64),
                                      _lib.stream_ptr()), "Tensor::contiguous")
    return out


class Tensor:
    """Dense N-d tensor with the reference's lazy permutation (Tensor_impl)."""

    def __init__(self, shape: Sequence[int] = (), dtype: int = Type.Double, device: Optional[int] = None,
                 init_zero: bool = True):
        dev = Device.default if device is None else device
        n = int(np.prod(shape)) if len(shape) else 1
        tdev = Device.torch_device(dev)
        self._storage = (torch.zeros if init_zero else torch.empty)(n, dtype=Type.to_torch(dtype), device=tdev)
        self._shape = [int(s) for s in shape]
        self._mapper = list(range(len(shape)))
        self._invmapper = list(range(len(shape)))
        self._contiguous = True

    # -------------------------------------------------------------- construction
    @staticmethod
    def from_torch(t: torch.Tensor) -> "Tensor":
        out = Tensor.__new__(Tensor)
        t = t.contiguous()
        out._storage = t.reshape(-1)
        out._shape = list(t.shape)
        out._mapper = list(range(t.dim()))
        out._invmapper = list(range(t.dim()))
        out._contiguous = True
        return out

    @staticmethod
    def from_numpy(a: np.ndarray, device: Optional[int] = None) -> "Tensor":
        dev = Device.default if device is None else device
        return Tensor.from_torch(torch.from_numpy(np.ascontiguousarray(a)).to(Device.torch_device(dev)))

    @staticmethod
    def from_dlpack(x) -> "Tensor":
        return Tensor.from_torch(torch.from_dlpack(x))

    def __dlpack__(self, stream=None):
        return self.to_torch().__dlpack__(stream=stream) if stream is not None else self.to_torch().__dlpack__()

    def __dlpack_device__(self):
        return self.to_torch().__dlpack_device__()

    def _view(self, shape, mapper, invmapper) -> "Tensor":
        out = Tensor.__new__(Tensor)
        out._storage = self._storage
        out._shape = list(shape)
        out._mapper = list(mapper)
        out._invmapper = list(invmapper)
        out._contiguous = all(m == i for i, m in enumerate(out._mapper))
        return out

    # -------------------------------------------------------------- metadata
    def shape(self) -> List[int]:
        return list(self._shape)

    def rank(self) -> int:
        return len(self._shape)

    def dtype(self) -> int:
        return Type.from_torch(self._storage.dtype)

    def dtype_str(self) -> str:
        return Type.getname(self.dtype())

    def device(self) -> int:
        return Device.from_torch(self._storage.device)

    def is_contiguous(self) -> bool:
        return self._contiguous

    def same_data(self, other: "Tensor") -> bool:
        return self._storage.data_ptr() == other._storage.data_ptr()

    def permute(self, *rnks) -> "Tensor":
        """Tensor_impl::permute (src/backend/Tensor_impl.cpp:38-86): metadata only."""
        if len(rnks) == 1 and isinstance(rnks[0], (list, tuple)):
            rnks = rnks[0]
        rnks = [int(r) for r in rnks]
        if len(rnks) != len(self._shape):
            raise CytnxError("reshape a tensor with a specify shape that does not match with the shape of the incident tensor.")
        if len(set(rnks)) != len(rnks):
            raise CytnxError("tensor permute with duplicated index.")
        if any(r < 0 or r >= len(rnks) for r in rnks):
            raise CytnxError("reshape a tensor with invalid rank index.")
        new_fwd = [self._mapper[r] for r in rnks]
        new_shape = [self._shape[r] for r in rnks]
        new_inv = [0] * len(rnks)
        for i, r in enumerate(rnks):
            new_inv[self._mapper[r]] = i
        return self._view(new_shape, new_fwd, new_inv)

    def permute_(self, *rnks) -> "Tensor":
        t = self.permute(*rnks)
        self._shape, self._mapper, self._invmapper, self._contiguous = t._shape, t._mapper, t._invmapper, t._contiguous
        return self

    def contiguous(self) -> "Tensor":
        """Tensor_impl::contiguous (include/backend/Tensor_impl.hpp:222-254)."""
        if self._contiguous:
            return self
        old_shape = [self._shape[self._invmapper[i]] for i in range(len(self._shape))]
        out = Tensor.__new__(Tensor)
        out._storage = device_permute(self._storage, old_shape, self._mapper)
        out._shape = list(self._shape)
        out._mapper = list(range(len(self._shape)))
        out._invmapper = list(range(len(self._shape)))
        out._contiguous = True
        return out

    def contiguous_(self) -> "Tensor":
        t = self.contiguous()
        self._storage, self._mapper, self._invmapper, self._contiguous = t._storage, t._mapper, t._invmapper, True
        return self

    def reshape(self, *shape) -> "Tensor":
        if len(shape) == 1 and isinstance(shape[0], (list, tuple)):
            shape = shape[0]
        shape = [int(s) for s in shape]
        n = int(np.prod(self._shape)) if self._shape else 1
        if shape.count(-1) > 1:
            raise CytnxError("[ERROR] reshape can have only one dimension specified as -1")
        if -1 in shape:
            k = int(np.prod([s for s in shape if s != -1])) if len(shape) > 1 else 1
            if k == 0 or n % k:
                raise CytnxError("[ERROR] unmatch size when reshape with undetermine dimension")
            shape[shape.index(-1)] = n // k
        if int(np.prod(shape)) != n:
            raise CytnxError("[ERROR] new shape does not match the number of elements.")
        base = self.contiguous()
        return base._view(shape, range(len(shape)), range(len(shape)))

    def reshape_(self, *shape) -> "Tensor":
        t = self.reshape(*shape)
        self._storage, self._shape, self._mapper, self._invmapper, self._contiguous = (
            t._storage, t._shape, t._mapper, t._invmapper, True)
        return self

    # -------------------------------------------------------------- data
    def to_torch(self) -> torch.Tensor:
        """The logical tensor as a torch view (materialised by the permute kernel if needed)."""
        c = self.contiguous()
        return c._storage.view(*c._shape) if c._shape else c._storage.view(())

    def numpy(self) -> np.ndarray:
        if self._contiguous:
            t = self._storage.view(*self._shape) if self._shape else self._storage.view(())
        elif self._storage.is_cuda:
            t = self.to_torch()
        else:
            # host tensors: metadata transpose through torch's strided view
            old_shape = [self._shape[self._invmapper[i]] for i in range(len(self._shape))]
            t = self._storage.view(*old_shape).permute(*self._mapper)
        return t.detach().cpu().numpy().copy()

    def to(self, device: int) -> "Tensor":
        out = self._view(self._shape, self._mapper, self._invmapper)
        out._storage = self._storage.to(Device.torch_device(device))
        return out

    def to_(self, device: int) -> "Tensor":
        self._storage = self._storage.to(Device.torch_device(device))
        return self

    def clone(self) -> "Tensor":
        out = self._view(self._shape, self._mapper, self._invmapper)
        out._storage = self._storage.clone()
        return out

    def astype(self, dtype: int) -> "Tensor":
        out = self._view(self._shape, self._mapper, self._invmapper)
        out._storage = self._storage.to(Type.to_torch(dtype))
        return out

    def __getitem__(self, key):
        return Tensor.from_torch(self.to_torch()[key])

    def __setitem__(self, key, value):
        """Element/slice assignment on the logical tensor (writes through to storage)."""
        if not self._contiguous:
            self.contiguous_()
        view = self._storage.view(*self._shape) if self._shape else self._storage.view(())
        if isinstance(value, Tensor):
            value = value.to_torch()
        view[key] = value

    def item(self):
        if self._storage.numel() != 1:
            raise CytnxError("[ERROR] item() requires a tensor with exactly one element")
        return self._storage.item()

    def __repr__(self):
        return f"Tensor(shape={self._shape}, dtype={self.dtype_str()}, device={self.device()})\n{self.numpy()}"


def arange(n, dtype: int = Type.Double, device: Optional[int] = None) -> Tensor:
    dev = Device.default if device is None else device
    return Tensor.from_torch(torch.arange(n, dtype=Type.to_torch(dtype), device=Device.torch_device(dev)))


def zeros(shape, dtype: int = Type.Double, device: Optional[int] = None) -> Tensor:
    return Tensor(shape, dtype, device)
