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
from typing import Optional, List, Sequence

import numpy as np
import torch

from . import _lib
from ._lib import CytnxError
from .core import Device, Tensor, Type, require_cuda
from .svd import Gesvd, Gesvd_truncate, Svd, Svd_truncate  # noqa: F401
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


_WHICH = {"SA": 0, "LA": 1, "LM": 2}


def Lanczos(Hop, Tin, method: Optional[str] = None, CvgCrit: Optional[float] = None, Maxiter: int = 10000,
            k: int = 1, is_V: bool = True, is_row: bool = False, max_krydim: int = 0, verbose: bool = False,
            which: Optional[str] = None, ncv: int = 0):
    """linalg::Lanczos in its two forms (src/linalg/Lanczos.cpp):
    * method form, ``Lanczos(Hop, Tin, method="Gnd", CvgCrit=1e-14, Maxiter=10000, ...)``: the
      ground state by the Lanczos_Gnd_Ut recurrence (:135-196);
    * which form, ``Lanczos(Hop, Tin, which="SA" | "LA" | "LM", Maxiter=10000, CvgCrit=0, k=1,
      is_V=True, ncv=0)``: the k extreme eigenpairs (:250-580; ARPACK there, a thick-restart
      Lanczos with full re-orthogonalisation on the device here)."""
    if which is not None:
        if method is not None:
            raise CytnxError("[ERROR][Lanczos] give either method or which, not both")
        return _lanczos_which(Hop, Tin, which, Maxiter, 0.0 if CvgCrit is None else CvgCrit, k, is_V, ncv, verbose)
    method = "Gnd" if method is None else method
    CvgCrit = 1.0e-14 if CvgCrit is None else CvgCrit
    if method == "ER":
        raise CytnxError("[ERROR][Lanczos] method 'ER' is not on this build's path; use method='Gnd' or the "
                         "which form (which='SA' gives the k lowest eigenpairs)")
    if method != "Gnd":
        raise CytnxError("[ERROR][Lanczos] Invalid Lanczos method, should be either 'ER' or 'Gnd'.")
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


def _lanczos_which(Hop, Tin, which, Maxiter, CvgCrit, k, is_V, ncv, verbose):
    """The which form (ctn_lanczos_which); argument checks and error texts of
    src/linalg/Lanczos.cpp:459-580."""
    if which not in _WHICH:
        raise CytnxError("[ERROR][Lanczos] 'which' should be 'LM', 'LA', 'SA'")
    if Hop.dtype() != Type.Double:
        raise CytnxError("[ERROR][Lanczos] the which form runs FP64 (Type.Double) operators on this build")
    nx = int(Hop.nx())
    if k < 1:
        raise CytnxError("[ERROR][Lanczos] k should be >0")
    if k > nx:
        raise CytnxError("[ERROR][Lanczos] k can only be up to total dimension of input vector D")
    if CvgCrit < 0:
        raise CytnxError("[ERROR][Lanczos] cvg_crit should be >= 0")
    if ncv != 0 and (ncv < 2 + k or ncv > nx):
        raise CytnxError("[ERROR][Lanczos] ncv should be 2+k<=ncv<=nx")
    if Maxiter < 1:
        raise CytnxError("[ERROR][Lanczos] Maxiter must be >= 1")
    is_uni = isinstance(Tin, UniTensor)
    if is_uni:
        if Tin.dtype() != Type.Double:
            raise CytnxError("[ERROR][Lanczos] Tin should have datatype consistent with Hop")
        v0 = Tin.contiguous()
        x0 = v0.flat_view()
    else:
        if Tin.dtype() != Type.Double:
            raise CytnxError("[ERROR][Lanczos] Tin should have datatype consistent with Hop")
        if len(Tin.shape()) != 1:
            raise CytnxError("[ERROR][Lanczos] Tin should be rank-1")
        v0 = Tin.contiguous()
        x0 = v0.to_torch().reshape(-1)
    n = x0.numel()
    if n != nx:
        raise CytnxError(f"[ERROR][Lanczos] Tin should have dimension consistent with Hop: [{nx}]")
    require_cuda(x0, "Lanczos")
    ncv_r = ncv if ncv else min(n, 2 * k + 10)
    if ncv_r <= k and ncv_r != n:
        raise CytnxError("[ERROR][Lanczos] ncv should be 2+k<=ncv<=nx")
    lib = _lib.lib()
    basis = torch.empty((ncv_r + 1) * n, dtype=torch.float64, device=x0.device)
    work = torch.empty(int(lib.ctn_lanczos_which_work_doubles(n, ncv_r)), dtype=torch.float64, device=x0.device)
    evecs = torch.empty(k * n, dtype=torch.float64, device=x0.device) if is_V else None
    evals = np.zeros(k, dtype=np.float64)
    cb = _Callback(Hop, v0, basis, work, n, is_uni)
    iters, nconv = ctypes.c_int(0), ctypes.c_int(0)
    st = lib.ctn_lanczos_which(cb.fn, None, x0.data_ptr(), n, _WHICH[which], int(k), int(ncv_r), int(Maxiter),
                               float(CvgCrit), basis.data_ptr(), work.data_ptr(), evals.ctypes.data_as(_lib.P_dbl),
                               evecs.data_ptr() if is_V else None, ctypes.byref(iters), ctypes.byref(nconv),
                               _lib.stream_ptr())
    if cb.err is not None:
        raise cb.err
    _lib.check(st, "Lanczos")
    if verbose and nconv.value < k:
        print(f"[WARNING][Lanczos]: Maximum number of iterations reached ({nconv.value} of {k} converged).")
    E = Tensor.from_numpy(evals.copy(), Device.cpu)
    if is_uni:
        out = [UniTensor(E, False, 0)]
        if is_V:
            out += [v0.with_flat(evecs[c * n:(c + 1) * n].clone()) for c in range(k)]
        return out
    out = [E]
    if is_V:
        out.append(Tensor.from_torch(evecs.view(n) if k == 1 else evecs.view(k, n)))
    return out


def Lanczos_Exp(Hop, v, tau, CvgCrit: float = 1.0e-14, Maxiter: int = 10000, verbose: bool = False):
    """exp(tau * Hop) v by Lanczos projection (linalg::Lanczos_Exp, src/linalg/Lanczos_Exp.cpp:
    264-453): the reference's recurrence, breakdown and stopping rules (ctn_lanczos_exp), on
    the device and for dense or block UniTensors / Tensors.  A real tau gives a Double
    result, a complex tau (real-time evolution) a ComplexDouble one."""
    if CvgCrit <= 0:
        raise CytnxError("[ERROR][Lanczos_Exp] converge criteria must >0")
    if Maxiter < 2:
        raise CytnxError("[ERROR][Lanczos_Exp] Maxiter must >1")
    if Hop.dtype() != Type.Double:
        raise CytnxError("[ERROR][Lanczos_Exp] FP64 (Type.Double) operators only on this build")
    tau = complex(tau)
    is_uni = isinstance(v, UniTensor)
    if is_uni:
        v0 = v.contiguous() if v.dtype() == Type.Double else v.astype(Type.Double).contiguous()
        x0 = v0.flat_view()
    else:
        v0 = v.contiguous().astype(Type.Double)
        x0 = v0.to_torch().reshape(-1)
    n = x0.numel()  # the vector's own size, as in the reference (no check against Hop.nx())
    require_cuda(x0, "Lanczos_Exp")
    lib = _lib.lib()
    mmax = min(int(Maxiter), n)
    basis = torch.empty(mmax * n, dtype=torch.float64, device=x0.device)
    work = torch.empty(int(lib.ctn_lanczos_exp_work_doubles(n, int(Maxiter))), dtype=torch.float64, device=x0.device)
    out_re = torch.empty(n, dtype=torch.float64, device=x0.device)
    out_im = torch.empty(n, dtype=torch.float64, device=x0.device) if tau.imag != 0 else None
    cb = _Callback(Hop, v0, basis, work, n, is_uni)
    iters = ctypes.c_int(0)
    st = lib.ctn_lanczos_exp(cb.fn, None, x0.data_ptr(), n, tau.real, tau.imag, float(CvgCrit), int(Maxiter),
                             basis.data_ptr(), work.data_ptr(), out_re.data_ptr(),
                             out_im.data_ptr() if out_im is not None else None, ctypes.byref(iters),
                             _lib.stream_ptr())
    if cb.err is not None:
        raise cb.err
    _lib.check(st, "Lanczos_Exp")
    if verbose:
        print(f"[Lanczos_Exp] Krylov dimension {iters.value}")
    flat = out_re if out_im is None else torch.complex(out_re, out_im)
    if is_uni:
        return v0.with_flat(flat)
    return Tensor.from_torch(flat.view(*v0.shape()))
