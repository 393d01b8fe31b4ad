"""Two-site effective Hamiltonian as a planned operator (the DMRG Lanczos hot path).

``TwoSiteHeff(L, M1, M2, R, psi)`` takes the network operands of
example/DMRG/dmrg_two_sites_U1.py:29-34 (leg orders psi[a,s1,s2,b], L[w,a,a'],
M1[w,w1,s1,s1'], M2[w1,w2,s2,s2'], R[w2,b,b']) and plans the matvec once in C++
(``ctn_heff2_plan_create``): block pairing, MPO folding and the grouped-GEMM task
tables are built on the host a single time; every ``matvec`` is then three launches.
It is a ``LinOp``: ``linalg.Lanczos(Hop=H, Tin=psi, method="Gnd")`` drives it through
the Python callback, and ``H.lanczos(psi)`` runs the same C++ driver with no Python
in the loop.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import BlockDesc, CytnxError, Heff2Desc
from .core import Device, Tensor, Type, require_cuda
from .network import LinOp
from .unitensor import UniTensor, UTenType, _desc, contract_plan_flops, layout_for, structure_only

_EPI = {0: "direct", 1: "staged", 2: "fragments"}  # tensor-core GEMM epilogue forms


def _plain_desc(u: UniTensor, keep):
    if u.uten_type() != UTenType.Block:
        raise CytnxError("[TwoSiteHeff] operands must be BlockUniTensors")
    u = u.contiguous()
    return u, _desc(u._layout, None, u._layout.itoi, u._layout.shapes, keep)


def plan_two_site(L: UniTensor, M1: UniTensor, M2: UniTensor, R: UniTensor, psi: UniTensor, keep: list):
    """Plan the two-site matvec on the host from the operands' block structure and the
    MPO values (no device data is read).  Returns (plan handle, contiguous operands,
    output bonds, output layout); ``keep`` collects the host arrays the plan was built from."""
    Lc, dL = _plain_desc(L, keep)
    M1c, dM1 = _plain_desc(M1, keep)
    M2c, dM2 = _plain_desc(M2, keep)
    Rc, dR = _plain_desc(R, keep)
    Pc, dP = _plain_desc(psi, keep)
    out_bonds = [Lc.bonds()[2], M1c.bonds()[3], M2c.bonds()[3], Rc.bonds()[2]]
    out_layout = layout_for(out_bonds)
    if not np.array_equal(out_layout.itoi, Pc._layout.itoi) or \
            not np.array_equal(out_layout.shapes, Pc._layout.shapes):
        raise CytnxError("[TwoSiteHeff] the output block structure differs from psi's")
    dO = _desc(out_layout, None, out_layout.itoi, out_layout.shapes, keep)
    m1h = M1c._data.detach().cpu().numpy().astype(np.float64)
    m2h = M2c._data.detach().cpu().numpy().astype(np.float64)
    keep += [m1h, m2h]
    desc = Heff2Desc(ctypes.pointer(dP), ctypes.pointer(dL), ctypes.pointer(dR), ctypes.pointer(dM1),
                     ctypes.pointer(dM2), ctypes.pointer(dO), m1h.ctypes.data, m2h.ctypes.data)
    h = ctypes.c_void_p()
    _lib.check(_lib.lib().ctn_heff2_plan_create(ctypes.byref(desc), ctypes.byref(h)), "TwoSiteHeff")
    return h.value, (Lc, M1c, M2c, Rc, Pc), out_bonds, out_layout


class MatvecGraph:
    """Replayable CUDA graph of TwoSiteHeff matvecs (TwoSiteHeff.capture)."""

    def __init__(self, op: "TwoSiteHeff", precision: str, graph, buffers):
        self._op, self._graph, self._buffers = op, graph, buffers
        self._prec = _lib.PRECISIONS[precision]
        self._replans = op._replans.get(self._prec, 0)

    def replay(self) -> None:
        if self._op._replans.get(self._prec, 0) != self._replans:
            raise CytnxError("[TwoSiteHeff] the captured matvec graph is stale: set_tiles re-planned its precision")
        self._graph.replay()


class TwoSiteHeff(LinOp):
    def __init__(self, L: UniTensor, M1: UniTensor, M2: UniTensor, R: UniTensor, psi: UniTensor,
                 precision: str = "fp64"):
        super().__init__("mv", psi.shape()[0] * psi.shape()[1] * psi.shape()[2] * psi.shape()[3], Type.Double,
                         psi.device())
        for t, nm in ((L, "L"), (M1, "M1"), (M2, "M2"), (R, "R"), (psi, "psi")):
            if t.dtype() != Type.Double:
                raise CytnxError(f"[TwoSiteHeff] {nm} must be float64")
        require_cuda(L._data, "TwoSiteHeff")
        keep: list = []
        self._h, (self.L, self.M1, self.M2, self.R, self.psi_t), self.out_bonds, self.out_layout = \
            plan_two_site(L, M1, M2, R, psi, keep)
        self._keep = keep
        self.n = int(_lib.lib().ctn_heff2_psi_elems(self._h))
        self.plan_flops = float(_lib.lib().ctn_heff2_flops(self._h))
        self._ws = {}
        self._bound = set()  # precisions whose environments are bound (each has its own workspace)
        self.precision = precision
        self._algo_flops = None
        self._replans = {}  # per precision: how often set_tiles re-planned it

    def __del__(self):
        try:
            _lib.lib().ctn_heff2_plan_destroy(self._h)
        except Exception:
            pass

    # ---------------------------------------------------------------- binding
    def bind(self, precision: Optional[str] = None) -> None:
        prec = _lib.PRECISIONS[(precision or self.precision).lower()]
        if prec in self._bound:
            return
        nbytes = int(_lib.lib().ctn_heff2_workspace_bytes(self._h, prec))
        ws = self._ws.get(prec)
        if ws is None:
            ws = torch.empty(nbytes, dtype=torch.uint8, device=self.L._data.device)
            self._ws[prec] = ws
        _lib.check(_lib.lib().ctn_heff2_set_env(self._h, self.L._data.data_ptr(), self.R._data.data_ptr(),
                                                ws.data_ptr(), prec, _lib.stream_ptr()), "TwoSiteHeff.set_env")
        self._bound.add(prec)

    # ---------------------------------------------------------------- matvec
    def apply_flat(self, x: torch.Tensor, y: torch.Tensor, precision: Optional[str] = None) -> None:
        prec = _lib.PRECISIONS[(precision or self.precision).lower()]
        self.bind(precision)
        _lib.check(_lib.lib().ctn_heff2_matvec(self._h, x.data_ptr(), y.data_ptr(), prec, _lib.stream_ptr()),
                   "TwoSiteHeff.matvec")

    def capture(self, x: torch.Tensor, y: torch.Tensor, precision: Optional[str] = None,
                count: int = 1) -> "MatvecGraph":
        """A CUDA graph of `count` matvecs y = H x on these buffers; ``replay()`` runs them again
        on the current stream without the per-launch host work (the matvec entry point only
        enqueues kernels and memsets on its stream, so it is capturable).  The graph reads the
        bound environments and the plan's device tables: it stays valid until set_tiles (or
        autotune) re-plans this precision, after which replay() raises."""
        prec = (precision or self.precision).lower()
        self.apply_flat(x, y, prec)  # binds, uploads the tables, sets kernel attributes
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            for _ in range(int(count)):
                self.apply_flat(x, y, prec)
        return MatvecGraph(self, prec, g, (x, y))

    def matvec(self, v: UniTensor) -> UniTensor:
        lbl = v.labels()
        x = v.contiguous().flat_view()
        if x.numel() != self.n:
            raise CytnxError("[TwoSiteHeff] psi has the wrong size")
        y = torch.empty_like(x)
        self.apply_flat(x, y)
        out = UniTensor._new_block(self.out_bonds, lbl, v.rowrank(), self.out_layout, [0, 1, 2, 3], y)
        return out

    # ---------------------------------------------------------------- tile autotuner
    def set_tiles(self, bn_step1: int, bn_step4: int, precision: Optional[str] = None) -> None:
        prec = _lib.PRECISIONS[(precision or self.precision).lower()]
        _lib.check(_lib.lib().ctn_heff2_set_tiles(self._h, prec, int(bn_step1), int(bn_step4)), "set_tiles")
        self._replans[prec] = self._replans.get(prec, 0) + 1  # invalidates captured graphs
        self._ws.pop(prec, None)
        self._bound.discard(prec)

    def autotune(self, precision: Optional[str] = None, step1=(128, 160, 192, 256, -192),
                 step4=(96, 128, 144, 160, 256, -128), reps: int = 5, epilogues=(0, 1, 2)) -> dict:
        """Pick the tensor-core tile width and epilogue form of steps 1 and 4 by timing them.

        The two GEMMs are independent kernels, so each is tuned with the other fixed:
        every width re-packs the operand panels (they depend on the width); for each
        width the epilogue forms (0 direct, 1 staged through shared memory, 2 TMEM fragments
        stored from registers) are timed
        with the per-phase CUDA-event profile (ctn_heff2_profile).  Negative widths are the
        2-CTA tiles (256 rows, cluster of two SMs); one of each step is a default candidate."""
        import ctypes as ct

        precision = (precision or self.precision).lower()
        if precision not in ("3xtf32", "bf16x3"):
            return {}
        prec = _lib.PRECISIONS[precision]
        x = self.psi_t.flat_view()
        y = torch.empty_like(x)

        def phase_ms(b1, b4, e1, e4):
            self.set_tiles(b1, b4, precision)
            self.bind(precision)
            _lib.check(_lib.lib().ctn_heff2_set_epilogue(self._h, prec, int(e1), int(e4)), "autotune")
            ms = (ct.c_double * 4)()
            nl = ct.c_int()
            _lib.check(_lib.lib().ctn_heff2_profile(self._h, x.data_ptr(), y.data_ptr(), prec, reps, ms, ct.byref(nl),
                                                   _lib.stream_ptr()), "autotune")
            return [ms[i] for i in range(4)]

        table = {"step1": {}, "step4": {}}
        for b1 in step1:
            for e in epilogues:
                table["step1"][(b1, e)] = phase_ms(b1, 128, e, -1)[1]
        best1 = min(table["step1"], key=table["step1"].get)
        for b4 in step4:
            for e in epilogues:
                table["step4"][(b4, e)] = phase_ms(best1[0], b4, best1[1], e)[3]
        best4 = min(table["step4"], key=table["step4"].get)
        self.set_tiles(best1[0], best4[0], precision)
        self.bind(precision)
        _lib.check(_lib.lib().ctn_heff2_set_epilogue(self._h, prec, best1[1], best4[1]), "autotune")
        return {"step1": best1[0], "step4": best4[0], "epilogue": [best1[1], best4[1]],
                "ms_step1": {f"{k[0]}/{_EPI[k[1]]}": v for k, v in table["step1"].items()},
                "ms_step4": {f"{k[0]}/{_EPI[k[1]]}": v for k, v in table["step4"].items()}}

    # ---------------------------------------------------------------- Lanczos without Python callbacks
    def lanczos(self, psi0: UniTensor, maxiter: int = 40, cvgcrit: float = 1e-14,
                precision: Optional[str] = None) -> Tuple[float, UniTensor, int]:
        prec = _lib.PRECISIONS[(precision or self.precision).lower()]
        self.bind(precision)
        x0 = psi0.contiguous().flat_view()
        n = self.n
        krylov = torch.empty((maxiter + 1) * n, dtype=torch.float64, device=x0.device)
        work = torch.empty(n + 8 + 1032 + maxiter + 64, dtype=torch.float64, device=x0.device)
        eig = torch.empty(n, dtype=torch.float64, device=x0.device)
        e = ctypes.c_double()
        it = ctypes.c_int()
        _lib.check(_lib.lib().ctn_heff2_lanczos_gnd(self._h, prec, x0.data_ptr(), maxiter, float(cvgcrit),
                                                    krylov.data_ptr(), work.data_ptr(), eig.data_ptr(),
                                                    ctypes.byref(e), ctypes.byref(it), _lib.stream_ptr()),
                   "TwoSiteHeff.lanczos")
        vec = UniTensor._new_block(self.out_bonds, psi0.labels(), psi0.rowrank(), self.out_layout, [0, 1, 2, 3], eig)
        return e.value, vec, it.value

    def lanczos_refined(self, psi0: UniTensor, precision: Optional[str] = None, krylov_dim: int = 20,
                        max_restarts: int = 200, tol: float = 1e-12) -> dict:
        """Restarted Lanczos: Krylov steps in ``precision``, one FP64 refinement matvec per
        restart (ctn_heff2_lanczos_refined).  Returns the FP64 Rayleigh quotient
        ``energy`` of the returned unit vector ``vec``, its FP64 eigen-residual
        ``residual`` = |H v - E v|, and the numbers of restarts and matvecs."""
        prec = _lib.PRECISIONS[(precision or self.precision).lower()]
        self.bind(precision)
        self.bind("fp64")
        x0 = psi0.contiguous().flat_view()
        n = self.n
        krylov = torch.empty(krylov_dim * n, dtype=torch.float64, device=x0.device)
        work = torch.empty(n + 3200 + 3 * krylov_dim, dtype=torch.float64, device=x0.device)
        eig = torch.empty(n, dtype=torch.float64, device=x0.device)
        e, r = ctypes.c_double(), ctypes.c_double()
        rs = ctypes.c_int()
        cnt = np.zeros(2, dtype=np.int64)
        _lib.check(_lib.lib().ctn_heff2_lanczos_refined(self._h, prec, x0.data_ptr(), int(krylov_dim),
                                                        int(max_restarts), float(tol), krylov.data_ptr(),
                                                        work.data_ptr(), eig.data_ptr(), ctypes.byref(e),
                                                        ctypes.byref(r), ctypes.byref(rs),
                                                        cnt.ctypes.data_as(_lib.P_i64), _lib.stream_ptr()),
                   "TwoSiteHeff.lanczos_refined")
        vec = UniTensor._new_block(self.out_bonds, psi0.labels(), psi0.rowrank(), self.out_layout, [0, 1, 2, 3], eig)
        return {"energy": e.value, "vec": vec, "residual": r.value, "restarts": rs.value,
                "matvecs_lo": int(cnt[0]), "matvecs_fp64": int(cnt[1])}

    # ---------------------------------------------------------------- accounting
    def algorithmic_flops(self) -> float:
        """Flops of the reference's block-pair GEMMs for one matvec in the order
        L -> M1 -> M2 -> R (2*m*n*k over every block pair each BlockUniTensor::contract
        step multiplies), counted on the host from the block structure."""
        if self._algo_flops is None:
            P = structure_only(self.psi_t.bonds(), ["a", "s1", "s2", "b"])
            Ls = structure_only(self.L.bonds(), ["w", "a", "ap"])
            M1s = structure_only(self.M1.bonds(), ["w", "w1", "s1", "s1p"])
            M2s = structure_only(self.M2.bonds(), ["w1", "w2", "s2", "s2p"])
            Rs = structure_only(self.R.bonds(), ["w2", "b", "bp"])
            f = 0.0
            f += contract_plan_flops(Ls, P)
            T1 = _struct_contract(Ls, P)
            f += contract_plan_flops(T1, M1s)
            T2 = _struct_contract(T1, M1s)
            f += contract_plan_flops(T2, M2s)
            T3 = _struct_contract(T2, M2s)
            f += contract_plan_flops(T3, Rs)
            self._algo_flops = f
        return self._algo_flops


def _struct_contract(A: UniTensor, B: UniTensor) -> UniTensor:
    comm = set(A.labels()) & set(B.labels())
    bonds = [b for b, l in zip(A.bonds(), A.labels()) if l not in comm] + \
        [b for b, l in zip(B.bonds(), B.labels()) if l not in comm]
    labels = [l for l in A.labels() if l not in comm] + [l for l in B.labels() if l not in comm]
    return structure_only(bonds, labels)
