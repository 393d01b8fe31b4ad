"""linalg: Lanczos (method "Gnd"), Tensordot, Vectordot, Tridiag, Norm, Svd_truncate.

* ``Lanczos(Hop, Tin, method="Gnd", CvgCrit, Maxiter, ...)`` -- Lanczos_Gnd_Ut /
  Lanczos_Gnd (src/linalg/Lanczos_Gnd_Ut.cpp:29-199, Lanczos_Gnd.cpp:16-134) run by the
  C++ driver ``ctn_lanczos_gnd`` on device vectors; the user's LinOp.matvec is called
  back with zero-copy UniTensor/Tensor views of the Krylov vectors.
* ``Tridiag`` -- the tridiagonal eigensolver of the library (implicit QL), same
  output convention as linalg::Tridiag (src/linalg/Tridiag.cpp:10-104).
* ``Tensordot`` -- src/linalg/Tensordot.cpp:165-207 through the planned contraction.
"""
from __future__ import annotations

import ctypes
from typing import List, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import CytnxError
from .core import Device, Tensor, Type, require_cuda
from .svd import Gesvd, Svd, Svd_truncate  # noqa: F401
from .unitensor import Contract, UniTensor, UTenType


def Tridiag(Diag, Sub_diag, is_V: bool = True, is_row: bool = True, throw_excp: bool = False):
    d = np.ascontiguousarray(Diag.numpy() if isinstance(Diag, Tensor) else Diag, dtype=np.float64).reshape(-1)
    e = np.ascontiguousarray(Sub_diag.numpy() if isinstance(Sub_diag, Tensor) else Sub_diag, dtype=np.float64).reshape(-1)
    n = len(d)
    if len(e) != max(n - 1, 0):
        raise CytnxError("[Tridiag] error, Sub_diag must have max(Diag.size()-1, 0) elements.")
    w = np.zeros(n)
    z = np.zeros((n, n)) if is_V else None
    if n:
        e2 = e if len(e) else np.zeros(1)
        _lib.check(_lib.lib().ctn_tridiag_eigh(n, d.ctypes.data_as(_lib.P_dbl), e2.ctypes.data_as(_lib.P_dbl),
                                               w.ctypes.data_as(_lib.P_dbl),
                                               z.ctypes.data_as(_lib.P_dbl) if is_V else None), "Tridiag")
    out = [Tensor.from_numpy(w, Device.cpu)]
    if is_V:
        out.append(Tensor.from_numpy(z if is_row else np.ascontiguousarray(z.T), Device.cpu))
    return out


def Vectordot(a: Tensor, b: Tensor, is_conj: bool = False) -> Tensor:
    x, y = a.to_torch().reshape(-1), b.to_torch().reshape(-1)
    if x.dtype == torch.float64 and x.is_cuda:
        out = torch.empty(1, dtype=torch.float64, device=x.device)
        _lib.check(_lib.lib().ctn_dot_f64(x.data_ptr(), y.data_ptr(), x.numel(), out.data_ptr(), _lib.stream_ptr()),
                   "Vectordot")
        return Tensor.from_torch(out)
    require_cuda(x, "Vectordot")
    return Tensor.from_torch(torch.dot(x.conj() if is_conj else x, y).reshape(1))


def Norm(t) -> Tensor:
    if isinstance(t, UniTensor):
        return t.Norm()
    x = t.to_torch().reshape(-1)
    require_cuda(x, "Norm")
    out = torch.empty(1, dtype=torch.float64, device=x.device)
    _lib.check(_lib.lib().ctn_nrm2_f64(x.data_ptr(), x.numel(), out.data_ptr(), _lib.stream_ptr()), "Norm")
    return Tensor.from_torch(out)


def Tensordot(Tl: Tensor, Tr: Tensor, idxl: Sequence[int], idxr: Sequence[int], cacheL: bool = False,
              cacheR: bool = False) -> Tensor:
    """Dense Tensordot via the contraction engine (free legs of Tl then of Tr)."""
    if len(idxl) != len(idxr):
        raise CytnxError("[ERROR][Tensordot] index lists must have the same length")
    la = [f"l{i}" for i in range(Tl.rank())]
    lb = [f"r{i}" for i in range(Tr.rank())]
    for k, (i, j) in enumerate(zip(idxl, idxr)):
        la[i] = lb[j] = f"c{k}"
    A = UniTensor(Tl, False, -1, la)
    B = UniTensor(Tr, False, -1, lb)
    out = Contract(A, B)
    # Contract orders common labels by name; the free legs keep Tl-then-Tr order either way
    return out.get_block_()


# ---------------------------------------------------------------- Lanczos
class _Callback:
    def __init__(self, Hop, template, krylov: torch.Tensor, work: torch.Tensor, n: int, is_uni: bool):
        self.Hop, self.template, self.krylov, self.work, self.n, self.is_uni = Hop, template, krylov, work, n, is_uni
        self.err = None
        self.base = krylov.data_ptr()
        self.fn = _lib.MATVEC_FN(self)

    def __call__(self, user, x, y, stream):
        try:
            i = (x - self.base) // (8 * self.n)
            xv = self.krylov[i * self.n: (i + 1) * self.n]
            if self.is_uni:
                v = self.template.with_flat(xv)
                out = self.Hop.matvec(v)
                if not isinstance(out, UniTensor):
                    raise CytnxError("[ERROR] LinOp.matvec(UniTensor) must return a UniTensor")
                if out.labels() != v.labels():
                    raise CytnxError("[ERROR] LinOp.matvec(UniTensor) -> UniTensor the output should have same labels and shape as input!")
                flat = out.contiguous().flat_view()
            else:
                v = Tensor.from_torch(xv.view(*self.template.shape()))
                out = self.Hop.matvec(v)
                flat = out.to_torch().reshape(-1)
            if flat.numel() != self.n or flat.dtype != torch.float64:
                raise CytnxError("[ERROR] LinOp.matvec output has the wrong size or dtype")
            self.work[: self.n].copy_(flat)
            return 0
        except Exception as e:  # surfaced after the driver returns
            self.err = e
            return 1


def Lanczos(Hop, Tin, method: str = "Gnd", CvgCrit: float = 1.0e-14, Maxiter: int = 10000, k: int = 1,
            is_V: bool = True, is_row: bool = False, max_krydim: int = 0, verbose: bool = False, which=None):
    """Ground state of a Hermitian LinOp (the 'Gnd' method of linalg::Lanczos)."""
    if which is not None or method not in ("Gnd",):
        raise CytnxError(f"[ERROR][Lanczos] method '{method if which is None else which}' is not on this build's "
                         "path; use method='Gnd'")
    if k != 1:
        raise CytnxError("[ERROR][Lanczos] method 'Gnd' returns only the ground state (k = 1)")
    if CvgCrit <= 0:
        raise CytnxError("[ERROR][Lanczos] converge criteria must >0")
    if Maxiter < 2:
        raise CytnxError("[ERROR][Lanczos] Maxiter must >1")
    is_uni = isinstance(Tin, UniTensor)
    if is_uni:
        if Tin.dtype() != Type.Double:
            Tin = Tin.astype(Type.Double)
        v0 = Tin.contiguous()
        x0 = v0.flat_view()
    else:
        v0 = Tin.contiguous().astype(Type.Double)
        x0 = v0.to_torch().reshape(-1)
    require_cuda(x0, "Lanczos")
    n = x0.numel()
    # Krylov storage (the reference keeps every psi_s when is_V): bounded by n and memory
    free, _ = torch.cuda.mem_get_info(x0.device)
    cap = max(2, int(0.6 * free // (8 * n)) - 2)
    maxiter = int(min(Maxiter, n, cap))
    maxiter = max(maxiter, 2)
    krylov = torch.empty((maxiter + 1) * n, dtype=torch.float64, device=x0.device)
    work = torch.empty(n + 8 + 1032 + maxiter + 64, dtype=torch.float64, device=x0.device)
    eig = torch.empty(n, dtype=torch.float64, device=x0.device)
    cb = _Callback(Hop, v0, krylov, work, n, is_uni)
    energy = ctypes.c_double(0.0)
    iters = ctypes.c_int(0)
    st = _lib.lib().ctn_lanczos_gnd(cb.fn, None, x0.data_ptr(), n, maxiter, float(CvgCrit), krylov.data_ptr(),
                                    work.data_ptr(), eig.data_ptr(), ctypes.byref(energy), ctypes.byref(iters),
                                    _lib.stream_ptr())
    if cb.err is not None:
        raise cb.err
    _lib.check(st, "Lanczos")
    E = Tensor.from_numpy(np.array([energy.value]), Device.cpu)
    out = [UniTensor(E, False, 0)] if is_uni else [E]
    if is_V:
        out.append(v0.with_flat(eig) if is_uni else Tensor.from_torch(eig.view(*v0.shape())))
    if verbose:
        print(f"[Lanczos] Gnd finished after {iters.value} iterations, E = {energy.value:.14f}")
    return out
