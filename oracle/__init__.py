"""CPU oracle for the cytnx hot path -- TEST INFRASTRUCTURE, never part of the product.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import this package, and only to check or to time the reference's CPU algorithm.

Contents (each restating the reference, Cytnx 1.1.1 source tree):

* ``permute``            -- ``src/backend/utils_internal_cpu/Movemem_cpu.cpp:152-191``
                            (C, ``oracle.c``), with the metadata rules of
                            ``src/backend/Tensor_impl.cpp:38-143``.
* ``enumerate_blocks``   -- ``src/BlockUniTensor.cpp:190-230`` + ``include/UniTensor.hpp:1139-1165``.
* ``BlockTensor.contract`` -- ``src/BlockUniTensor.cpp:777-1235`` (non-MKL branch :1180-1223),
                            label intersection ``src/utils/vec_intersect.cpp:35-51`` (common
                            labels sorted), output bonds/labels/rowrank ``:1028-1050``.
* ``lanczos_gnd_ut``     -- ``src/linalg/Lanczos_Gnd_Ut.cpp:29-162`` with ``linalg::Tridiag``
                            = LAPACKE_dstev (``src/backend/linalg_internal_cpu/Tridiag_internal.cpp:9-42``).
* ``tensordot``          -- ``src/linalg/Tensordot.cpp:29-110`` (permute -> reshape -> Matmul).

BLAS/LAPACK: the container's OpenBLAS bundled with scipy (``scipy_dgemm_``,
``scipy_zgemm_``, ``scipy_LAPACKE_dstev``); the reference links OpenBLAS 0.3.33 /
liblapacke 3.11.0 (pixi.lock), the same published routines.
"""
from __future__ import annotations

import ctypes
import glob
import os
import subprocess
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        os.makedirs(BUILD, exist_ok=True)
        subprocess.check_call(["gcc", "-O2", "-fPIC", "-shared", "-std=c11", src, "-o", LIB])
    return LIB


_lib = None
_blas = None


def _openblas():
    global _blas
    if _blas is None:
        import scipy

        libdir = os.path.join(os.path.dirname(os.path.dirname(scipy.__file__)), "scipy.libs")
        cands = sorted(glob.glob(os.path.join(libdir, "libscipy_openblas*.so")))
        if not cands:
            raise RuntimeError("scipy's bundled OpenBLAS not found")
        _blas = ctypes.CDLL(cands[0])
    return _blas


def set_threads(n: int) -> None:
    b = _openblas()
    fn = getattr(b, "scipy_openblas_set_num_threads", None)
    if fn is not None:
        fn.argtypes = [ctypes.c_int]
        fn(int(n))


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = ctypes.CDLL(LIB)
        b = _openblas()
        _lib.orc_set_blas.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        _lib.orc_set_blas(ctypes.cast(b.scipy_dgemm_, ctypes.c_void_p),
                          ctypes.cast(b.scipy_zgemm_, ctypes.c_void_p))
        _lib.orc_permute.restype = ctypes.c_int
        _lib.orc_blocks_enumerate.restype = ctypes.c_int64
        _lib.orc_bs_contract.restype = ctypes.c_int
        _lib.orc_bs_contract_ex.restype = ctypes.c_int
    return _lib


def _u64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ------------------------------------------------------------------ permute
def permute(arr: np.ndarray, mapper: Sequence[int]) -> np.ndarray:
    """Tensor.permute(mapper).contiguous() on a row-major array (Movemem_cpu.cpp:152-191)."""
    arr = np.ascontiguousarray(arr)
    rank = arr.ndim
    mapper = [int(m) for m in mapper]
    inv = [0] * rank
    for i, m in enumerate(mapper):
        inv[m] = i
    out = np.empty([arr.shape[m] for m in mapper], dtype=arr.dtype)
    if arr.size == 0:
        return out
    rc = lib().orc_permute(_p(arr), _p(out), ctypes.c_int64(arr.itemsize), ctypes.c_int(rank),
                           _p(_u64(arr.shape)), _p(_u64(mapper)), _p(_u64(inv)))
    if rc:
        raise RuntimeError("orc_permute failed")
    return out


def permute_meta(shape, mapper, invmapper, rnks):
    """Tensor_impl::permute metadata rule (src/backend/Tensor_impl.cpp:38-86)."""
    new_fwd = [mapper[r] for r in rnks]
    new_shape = [shape[r] for r in rnks]
    new_inv = [0] * len(rnks)
    for i, r in enumerate(rnks):
        new_inv[mapper[r]] = i
    conti = all(new_fwd[i] == i for i in range(len(rnks)))
    return new_shape, new_fwd, new_inv, conti


# ------------------------------------------------------------- blocks
class Bond:
    """(type, qnums[nq][nsym], degs[nq], syms[(stype, n)]) -- include/Bond.hpp:41-71."""

    def __init__(self, btype: int, qnums, degs, syms=None):
        self.type = int(btype)
        self.qnums = np.asarray(qnums, dtype=np.int64).reshape(len(degs), -1)
        self.degs = np.asarray(degs, dtype=np.int64)
        nsym = self.qnums.shape[1]
        self.syms = list(syms) if syms is not None else [(-1, 1)] * nsym

    def redirect(self):
        return Bond(-self.type, self.qnums, self.degs, self.syms)


def enumerate_blocks(bonds: Sequence[Bond]) -> np.ndarray:
    rank = len(bonds)
    nsym = bonds[0].qnums.shape[1]
    stype = np.array([s[0] for s in bonds[0].syms], dtype=np.int32)
    symn = np.array([s[1] for s in bonds[0].syms], dtype=np.int64)
    btypes = np.array([b.type for b in bonds], dtype=np.int32)
    nqs = _i64([len(b.degs) for b in bonds])
    tabs = [np.ascontiguousarray(b.qnums, dtype=np.int64) for b in bonds]
    ptrs = (ctypes.c_void_p * rank)(*[t.ctypes.data for t in tabs])
    cap = int(np.prod([max(1, n) for n in nqs]))
    out = np.zeros((cap, rank), dtype=np.int64)
    n = lib().orc_blocks_enumerate(ctypes.c_int(rank), ctypes.c_int(nsym), _p(stype), _p(symn),
                                   _p(btypes), _p(nqs), ptrs, _p(out), ctypes.c_int64(cap))
    if n < 0:
        raise RuntimeError("enumeration overflow")
    return out[:n].copy()


class _Layout(ctypes.Structure):
    _fields_ = [("rank", ctypes.c_int), ("nblocks", ctypes.c_int64), ("itoi", ctypes.c_void_p),
                ("shapes", ctypes.c_void_p), ("offs", ctypes.c_void_p)]


class BlockTensor:
    """Minimal BlockUniTensor: bonds, labels, rowrank, itoi, and numpy blocks."""

    def __init__(self, bonds: List[Bond], labels: List[str], rowrank: int, itoi=None,
                 blocks=None, dtype=np.float64):
        self.bonds = bonds
        self.labels = [str(l) for l in labels]
        self.rowrank = rowrank
        self.itoi = enumerate_blocks(bonds) if itoi is None else np.asarray(itoi, dtype=np.int64)
        if blocks is None:
            blocks = [np.zeros(self.block_shape(t), dtype=dtype) for t in self.itoi]
        self.blocks = blocks

    def block_shape(self, tup):
        return tuple(int(self.bonds[i].degs[q]) for i, q in enumerate(tup))

    @property
    def dtype(self):
        return self.blocks[0].dtype if self.blocks else np.float64

    def flat(self):
        return np.concatenate([b.ravel() for b in self.blocks]) if self.blocks else np.zeros(0)

    def _layout(self, keep):
        shapes = _i64([b.shape for b in self.blocks]).reshape(len(self.blocks), len(self.bonds))
        sizes = shapes.prod(axis=1) if len(self.blocks) else np.zeros(0, np.int64)
        offs = _i64(np.concatenate([[0], np.cumsum(sizes)[:-1]])) if len(sizes) else _i64([])
        itoi = _i64(self.itoi).reshape(len(self.blocks), len(self.bonds))
        keep += [shapes, offs, itoi]
        return _Layout(len(self.bonds), len(self.blocks), itoi.ctypes.data, shapes.ctypes.data,
                       offs.ctypes.data)

    def permute(self, mapper: Sequence[int], rowrank: Optional[int] = None) -> "BlockTensor":
        """BlockUniTensor::permute (src/BlockUniTensor.cpp:588-632): bonds, labels,
        each qindex tuple, and each block are permuted by the same mapper."""
        mapper = list(mapper)
        return BlockTensor([self.bonds[m] for m in mapper], [self.labels[m] for m in mapper],
                           self.rowrank if rowrank is None else rowrank,
                           self.itoi[:, mapper] if len(self.itoi) else self.itoi,
                           [permute(b, mapper) for b in self.blocks])

    def contract(self, rhs: "BlockTensor", stride: int = 1, offset: int = 0, out: "BlockTensor" = None,
                 flops: list = None) -> "BlockTensor":
        """BlockUniTensor::contract.  ``stride`` > 1 multiplies only every stride-th block
        pair (from ``offset``) into ``out`` (a bounded sample of the work for CPU timings);
        ``stride`` 0 only counts.  ``flops`` (a list) receives 2*M*N*K of the pairs taken."""
        comm = sorted(set(self.labels) & set(rhs.labels))
        c1 = [self.labels.index(l) for l in comm]
        c2 = [rhs.labels.index(l) for l in comm]
        if not comm:
            raise NotImplementedError("outer product is not on the oracle's path")
        for a, b in zip(c1, c2):
            if self.bonds[a].type + rhs.bonds[b].type != 0:
                raise ValueError("BRA can only be contracted with KET")
        n1 = [i for i in range(len(self.labels)) if i not in c1]
        n2 = [i for i in range(len(rhs.labels)) if i not in c2]
        dt = np.result_type(self.dtype, rhs.dtype)
        if len(n1) + len(n2) == 0:
            # all legs contracted: sum over matching blocks of vectordot (:898-928)
            lp = self.permute(c1)
            rp = rhs.permute(c2)
            s = np.zeros((), dtype=dt)
            for b in range(len(lp.blocks)):
                for a in range(len(rp.blocks)):
                    if np.array_equal(lp.itoi[b], rp.itoi[a]):
                        s = s + np.dot(lp.blocks[b].ravel(), rp.blocks[a].ravel())
            return s
        out_bonds = [self.bonds[i] for i in n1] + [rhs.bonds[i] for i in n2]
        out_labels = [self.labels[i] for i in n1] + [rhs.labels[i] for i in n2]
        rowrank = self.rowrank + rhs.rowrank - sum(1 for i in c1 if i < self.rowrank) \
            - sum(1 for i in c2 if i < rhs.rowrank)
        reuse = out is not None
        if not reuse:
            out = BlockTensor(out_bonds, out_labels, rowrank, dtype=dt)
        code = {np.dtype(np.float64): 3, np.dtype(np.complex128): 1}[np.dtype(dt)]
        L = self if self.dtype == dt else self.astype(dt)
        R = rhs if rhs.dtype == dt else rhs.astype(dt)
        keep = []
        ldat = self._flat_cache(L)
        rdat = rhs._flat_cache(R)
        if reuse:
            odat = out._odat
        else:
            odat = np.zeros(sum(b.size for b in out.blocks), dtype=dt)
        fl = ctypes.c_double(0.0)
        rc = lib().orc_bs_contract_ex(ctypes.c_int(code), L._layout(keep), _p(ldat),
                                      R._layout(keep), _p(rdat), ctypes.c_int(len(comm)),
                                      _p(_i64(c1)), _p(_i64(c2)), out._layout(keep), _p(odat),
                                      ctypes.c_int64(stride), ctypes.c_int64(offset), ctypes.byref(fl))
        if rc:
            raise RuntimeError(f"orc_bs_contract failed ({rc})")
        if flops is not None:
            flops.append(fl.value)
        if not reuse:
            pos = 0
            for i, b in enumerate(out.blocks):
                out.blocks[i] = odat[pos:pos + b.size].reshape(b.shape)
                pos += b.size
            out._odat = odat
        return out

    def contract_flops(self, rhs: "BlockTensor") -> float:
        """2*M*N*K summed over the block pairs BlockUniTensor::contract multiplies."""
        fl = []
        self.contract(rhs, stride=0, flops=fl)
        return fl[0]

    def _flat_cache(self, conv):
        """Contiguous flat data of ``conv`` (this tensor or its dtype conversion).  When
        every block is still a view into the one buffer it was made from (a contract
        result, or ``from_flat``), that buffer is used as it is."""
        od = getattr(self, "_odat", None)
        if conv is self and od is not None and all(b.base is od for b in self.blocks):
            return od
        return np.ascontiguousarray(conv.flat())

    @classmethod
    def from_flat(cls, bonds, labels, rowrank, itoi, flat) -> "BlockTensor":
        """Blocks as views into ``flat`` (back to back in ``itoi`` order, row-major)."""
        t = cls(bonds, labels, rowrank, itoi, blocks=[])
        flat = np.ascontiguousarray(flat)
        blocks, pos = [], 0
        for tup in t.itoi:
            shp = t.block_shape(tup)
            n = int(np.prod(shp))
            blocks.append(flat[pos:pos + n].reshape(shp))
            pos += n
        if pos != flat.size:
            raise ValueError("flat data size does not match the blocks")
        t.blocks = blocks
        t._odat = flat
        return t

    def astype(self, dt):
        return BlockTensor(self.bonds, self.labels, self.rowrank, self.itoi,
                           [b.astype(dt) for b in self.blocks])

    def relabel(self, labels):
        return BlockTensor(self.bonds, list(labels), self.rowrank, self.itoi, self.blocks)

    def norm(self):
        return float(np.sqrt(sum(float(np.vdot(b, b).real) for b in self.blocks)))

    def dense(self) -> np.ndarray:
        """Dense array with every block placed at its sector offsets (for checks)."""
        offs = [np.concatenate([[0], np.cumsum(b.degs)[:-1]]) for b in self.bonds]
        full = np.zeros([int(b.degs.sum()) for b in self.bonds], dtype=self.dtype)
        for t, blk in zip(self.itoi, self.blocks):
            sl = tuple(slice(offs[i][q], offs[i][q] + self.bonds[i].degs[q]) for i, q in enumerate(t))
            full[sl] = blk
        return full


# ------------------------------------------------------------------ Lanczos
def dstev(d: np.ndarray, e: np.ndarray):
    """LAPACKE_dstev('V') as called by Tridiag_internal_d (Tridiag_internal.cpp:9-42).
    Returns (eigenvalues ascending, eigenvectors as rows)."""
    b = _openblas()
    fn = b.scipy_LAPACKE_dstev
    fn.restype = ctypes.c_int
    n = len(d)
    w = np.ascontiguousarray(d, dtype=np.float64).copy()
    ee = np.ascontiguousarray(e, dtype=np.float64).copy() if n > 1 else np.zeros(1)
    z = np.zeros((n, n), dtype=np.float64)  # column-major: z[:, j] stored as row j in C order
    info = fn(ctypes.c_int(102), ctypes.c_char(b"V"), ctypes.c_int(n), _p(w), _p(ee), _p(z),
              ctypes.c_int(n))
    if info != 0:
        raise RuntimeError(f"dstev info={info}")
    # col-major Z with ldz=n read as C-order array gives Z^T: row j = eigenvector j (is_row=True)
    return w, z


def lanczos_gnd_ut(matvec, psi0: np.ndarray, cvgcrit: float, maxiter: int):
    """Lanczos_Gnd_Ut (src/linalg/Lanczos_Gnd_Ut.cpp:29-162) on flat float64 vectors.

    matvec maps a flat vector to a flat vector (the block-sparse H_eff of the
    caller).  Returns (energy, eigenvector, number of iterations done)."""
    psi_1 = psi0 / np.linalg.norm(psi0)
    psi_s = [psi_1]
    new_psi = matvec(psi_1)
    alpha = float(np.dot(new_psi, psi_1))
    As = [alpha]
    new_psi = new_psi - alpha * psi_1
    beta = float(np.linalg.norm(new_psi))
    Bs = [beta]
    psi_0 = psi_1
    new_psi = new_psi / beta
    psi_1 = new_psi
    psi_s.append(psi_1)
    E = alpha
    evals, evecs = np.array([alpha]), np.ones((1, 1))
    it = 1
    for i in range(1, maxiter):
        it = i + 1
        new_psi = matvec(psi_1)
        alpha = float(np.dot(new_psi, psi_1))
        As.append(alpha)
        new_psi = new_psi - (alpha * psi_1 + beta * psi_0)
        evals, evecs = dstev(np.array(As), np.array(Bs))
        beta = float(np.linalg.norm(new_psi))
        Bs.append(beta)
        if beta == 0:
            break
        psi_0 = psi_1
        psi_1 = new_psi / beta
        psi_s.append(psi_1)
        ediff = abs(E - evals[0])
        if ediff < cvgcrit:
            break
        E = evals[0]
    kry = evecs[0]
    ev = kry[0] * psi_s[0]
    for n in range(1, len(evals)):
        ev = ev + kry[n] * psi_s[n]
    return float(evals[0]), ev, it


# ------------------------------------------------------------------ dense
def tensordot(a: np.ndarray, b: np.ndarray, idxl: Sequence[int], idxr: Sequence[int]) -> np.ndarray:
    """_Tensordot_generic (src/linalg/Tensordot.cpp:29-110): permute both operands to
    (free ++ contracted) / (contracted ++ free), reshape, Matmul."""
    nl = [i for i in range(a.ndim) if i not in idxl]
    nr = [i for i in range(b.ndim) if i not in idxr]
    am = permute(a, nl + list(idxl))
    bm = permute(b, list(idxr) + nr)
    k = int(np.prod([a.shape[i] for i in idxl])) if idxl else 1
    out = am.reshape(-1, k) @ bm.reshape(k, -1)
    return out.reshape([a.shape[i] for i in nl] + [b.shape[i] for i in nr])
