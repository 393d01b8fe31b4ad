"""Reader/writer for the cytnx binary object format (``.cytnx`` / ``.cytn``).

The layout follows the reference's save/load code:

* UniTensor: ``src/UniTensor.cpp:68-143`` (magic 555 legacy, 556 + u32 version),
  Block dispatch ``src/BlockUniTensor.cpp:1618-1662``, Dense dispatch
  ``src/DenseUniTensor.cpp:1314-1324``.
* Bond: ``src/Bond.cpp:500-607`` (magic 666, ver 0 = plain dim, ver 1 = qnums + degs).
* Symmetry: ``src/Symmetry.cpp:257-275`` (magic 777, i32 stype, i32 n).
* Tensor: ``src/Tensor.cpp:472-541`` (magic 888 legacy, 889 + u32 version; rank,
  contiguous flag, shape, mapper, invmapper, then Storage).
* Storage: ``src/backend/Storage.cpp:161-330`` (magic 999, u64 size, u32 dtype,
  i32 device, raw data).

Objects are returned as plain dictionaries of numpy arrays so the module has no
dependency on torch or on the CUDA library; ``cytnx_b200.UniTensor.Load`` builds
device tensors from them.
"""
from __future__ import annotations

import struct
from typing import Any, BinaryIO, Dict, List

import numpy as np

# dtype ids of the reference (include/Type.hpp:177-179): index into the type list.
DTYPE_NP = {
    1: np.complex128,
    2: np.complex64,
    3: np.float64,
    4: np.float32,
    5: np.int64,
    6: np.uint64,
    7: np.int32,
    8: np.uint32,
    9: np.int16,
    10: np.uint16,
    11: np.bool_,
}
NP_DTYPE = {np.dtype(v): k for k, v in DTYPE_NP.items()}

UTEN_DENSE = 0
UTEN_BLOCK = 2


class FormatError(ValueError):
    pass


class _Reader:
    def __init__(self, f: BinaryIO):
        self.f = f

    def read(self, fmt: str):
        n = struct.calcsize(fmt)
        b = self.f.read(n)
        if len(b) != n:
            raise FormatError("unexpected end of file")
        return struct.unpack("<" + fmt, b)

    def u32(self):
        return self.read("I")[0]

    def i32(self):
        return self.read("i")[0]

    def u64(self):
        return self.read("Q")[0]

    def i64(self):
        return self.read("q")[0]

    def boolean(self):
        return bool(self.read("?")[0])

    def raw(self, n: int) -> bytes:
        b = self.f.read(n)
        if len(b) != n:
            raise FormatError("unexpected end of file")
        return b


def _read_symmetry(r: _Reader) -> Dict[str, int]:
    if r.u32() != 777:
        raise FormatError("not a cytnx Symmetry")
    stype = r.i32()
    n = r.i32()
    return {"stype": stype, "n": n}


def _read_bond(r: _Reader) -> Dict[str, Any]:
    if r.u32() != 666:
        raise FormatError("not a cytnx Bond")
    ver = r.i32()
    dim_or_nq = r.u64()
    btype = r.i32()
    nsym = r.u64()
    bond: Dict[str, Any] = {"type": btype, "nsym": nsym}
    if ver == 0:
        bond["dim"] = dim_or_nq
        if nsym:
            q = np.frombuffer(r.raw(8 * nsym * dim_or_nq), dtype="<i8").reshape(dim_or_nq, nsym)
            bond["qnums"] = q.copy()
            bond["degs"] = np.ones(dim_or_nq, dtype=np.uint64)
        else:
            bond["qnums"] = np.zeros((0, 0), dtype=np.int64)
            bond["degs"] = np.zeros(0, dtype=np.uint64)
    else:
        nq = dim_or_nq
        q = np.frombuffer(r.raw(8 * nsym * nq), dtype="<i8").reshape(nq, nsym)
        degs = np.frombuffer(r.raw(8 * nq), dtype="<u8")
        bond["qnums"] = q.copy()
        bond["degs"] = degs.copy()
        bond["dim"] = int(degs.sum())
    bond["syms"] = [_read_symmetry(r) for _ in range(nsym)]
    return bond


def _read_storage(r: _Reader) -> np.ndarray:
    if r.u32() != 999:
        raise FormatError("not a cytnx Storage")
    size = r.u64()
    dtype = r.u32()
    _device = r.i32()
    if dtype not in DTYPE_NP:
        raise FormatError(f"unsupported storage dtype id {dtype}")
    npdt = np.dtype(DTYPE_NP[dtype]).newbyteorder("<")
    return np.frombuffer(r.raw(npdt.itemsize * size), dtype=npdt).copy()


def _read_tensor(r: _Reader) -> np.ndarray:
    magic = r.u32()
    if magic == 889:
        if r.u32() != 1:
            raise FormatError("unsupported Tensor file version")
    elif magic != 888:
        raise FormatError("not a cytnx Tensor")
    rank = r.u64()
    _conti = r.u64()
    if rank:
        shape = list(r.read(f"{rank}Q"))
        mapper = list(r.read(f"{rank}Q"))
        invmapper = list(r.read(f"{rank}Q"))
    else:
        shape, mapper, invmapper = [], [], []
    data = _read_storage(r)
    # The storage holds the physical (pre-permute) order: old_shape[i] = shape[invmapper[i]]
    # (include/backend/Tensor_impl.hpp:244-247); the logical view is its transpose by mapper.
    old_shape = [shape[invmapper[i]] for i in range(rank)]
    arr = data.reshape(old_shape) if rank else data.reshape(())
    if rank:
        arr = np.ascontiguousarray(arr.transpose(mapper))
    return arr


def read_tensor(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        return _read_tensor(_Reader(f))


def read_unitensor(path: str) -> Dict[str, Any]:
    """Parse a saved UniTensor into a dict with bonds, labels, and blocks (numpy)."""
    with open(path, "rb") as f:
        r = _Reader(f)
        magic = r.u32()
        version = 0
        if magic == 556:
            version = r.u32()
            if version != 1:
                raise FormatError("unsupported UniTensor file version")
        elif magic != 555:
            raise FormatError("not a cytnx UniTensor")
        utype = r.i32()
        braket = r.boolean()
        tag = r.boolean()
        diag = r.boolean()
        rowrank = r.i64()
        lname = r.u32()
        name = r.raw(lname).decode() if lname else ""
        rank = r.u64()
        lens = [r.u64() for _ in range(rank)]
        labels = [r.raw(n).decode() for n in lens]
        bonds = [_read_bond(r) for _ in range(rank)]
        out: Dict[str, Any] = {
            "uten_type": utype,
            "is_braket_form": braket,
            "is_tag": tag,
            "is_diag": diag,
            "rowrank": rowrank,
            "name": name,
            "labels": labels,
            "bonds": bonds,
        }
        if utype == UTEN_BLOCK:
            if rank == 0 and version > 0:
                nsyms = r.u64()
                out["syms"] = [_read_symmetry(r) for _ in range(nsyms)]
            nblocks = r.u64()
            itoi = np.zeros((nblocks, rank), dtype=np.int64)
            for b in range(nblocks):
                if rank:
                    itoi[b] = r.read(f"{rank}Q")
            out["itoi"] = itoi
            out["blocks"] = [_read_tensor(r) for _ in range(nblocks)]
        elif utype == UTEN_DENSE:
            out["block"] = _read_tensor(r)
        else:
            raise FormatError(f"unsupported UniTensor type {utype}")
        rest = f.read()
        if rest:
            raise FormatError(f"{len(rest)} trailing bytes")
        return out


# ---------------------------------------------------------------- writer
def _w(f: BinaryIO, fmt: str, *vals):
    f.write(struct.pack("<" + fmt, *vals))


def _write_symmetry(f, sym):
    _w(f, "Iii", 777, sym["stype"], sym["n"])


def _write_bond(f, bond):
    _w(f, "I", 666)
    qn = np.asarray(bond["qnums"], dtype="<i8")
    degs = np.asarray(bond["degs"], dtype="<u8")
    if len(degs):
        _w(f, "iQ", 1, len(degs))
    else:
        _w(f, "iQ", 0, int(bond["dim"]))
    _w(f, "iQ", int(bond["type"]), int(bond["nsym"]))
    if len(degs):
        f.write(qn.tobytes())
        f.write(degs.tobytes())
    for s in bond["syms"]:
        _write_symmetry(f, s)


def _write_tensor(f, arr: np.ndarray):
    arr = np.ascontiguousarray(arr)
    _w(f, "II", 889, 1)
    rank = arr.ndim
    _w(f, "QQ", rank, 1)
    if rank:
        _w(f, f"{rank}Q", *arr.shape)
        _w(f, f"{rank}Q", *range(rank))
        _w(f, f"{rank}Q", *range(rank))
    dt = NP_DTYPE[arr.dtype]
    _w(f, "IQIi", 999, arr.size, dt, -1)
    f.write(arr.astype(arr.dtype.newbyteorder("<"), copy=False).tobytes())


def write_unitensor(path: str, ut: Dict[str, Any]) -> None:
    """Write the versioned (556/v1) layout that the reference's loader accepts."""
    with open(path, "wb") as f:
        _w(f, "II", 556, 1)
        _w(f, "i", ut["uten_type"])
        _w(f, "???", ut["is_braket_form"], ut["is_tag"], ut["is_diag"])
        _w(f, "q", ut["rowrank"])
        name = ut.get("name", "").encode()
        _w(f, "I", len(name))
        f.write(name)
        labels: List[str] = ut["labels"]
        _w(f, "Q", len(labels))
        for l in labels:
            _w(f, "Q", len(l.encode()))
        for l in labels:
            f.write(l.encode())
        for b in ut["bonds"]:
            _write_bond(f, b)
        if ut["uten_type"] == UTEN_BLOCK:
            if not labels:
                syms = ut.get("syms", [])
                _w(f, "Q", len(syms))
                for s in syms:
                    _write_symmetry(f, s)
            blocks = ut["blocks"]
            _w(f, "Q", len(blocks))
            for it in np.asarray(ut["itoi"], dtype="<u8").reshape(len(blocks), -1):
                if labels:
                    f.write(it.tobytes())
            for blk in blocks:
                _write_tensor(f, blk)
        else:
            _write_tensor(f, ut["block"])
