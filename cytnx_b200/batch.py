"""Many independent two-site H_eff problems applied as one batch.

``BatchedTwoSiteHeff(problems)`` plans every problem with the two-site planner
(``plan_two_site``), then concatenates their split-precision tables in C++
(``ctn_heff2_batch_create``): one matvec of the whole batch is one pack launch, one
persistent tcgen05 grouped-GEMM launch over the tiles of every problem's step-1
groups, one MPO-fold launch and one persistent grouped-GEMM launch for step 4 -- the
same four launches whatever the number of problems or the spread of their block
sizes.  The sequence has no host synchronisation, so ``capture`` records it in a CUDA
graph that ``replay`` launches with a single call.

Vectors and environments of all problems live in shared flat device buffers
(FP32 by default, FP64 with ``fp32=False``) at the offsets ``psi_offsets`` /
``L_offsets`` / ``R_offsets``; each problem's slice holds its blocks in the
BlockUniTensor order of its own ``psi`` / ``L`` / ``R``.

The per-problem operation is the network of example/DMRG/dmrg_two_sites_U1.py:18-23
(psi[a,s1,s2,b], L[w,a,a'], M1[w,w1,s1,s1'], M2[w1,w2,s2,s2'], R[w2,b,b']); the
reference applies it one problem at a time through Network::Launch.
"""
from __future__ import annotations

import ctypes
import os
from concurrent.futures import ThreadPoolExecutor
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import CytnxError
from .heff import plan_two_site
from .unitensor import UniTensor

_ALIGN = 32  # element alignment of every problem's slice (128 bytes in FP32)


def _aligned_offsets(sizes: Sequence[int]) -> Tuple[np.ndarray, int]:
    offs = np.zeros(len(sizes), dtype=np.int64)
    o = 0
    for i, n in enumerate(sizes):
        offs[i] = o
        o += (int(n) + _ALIGN - 1) // _ALIGN * _ALIGN
    return offs, o


class BatchedTwoSiteHeff:
    """``problems``: sequence of (L, M1, M2, R, psi) BlockUniTensors.  Only their block
    structure and the MPO values are read (structure-only tensors are fine)."""

    def __init__(self, problems: Sequence[Tuple[UniTensor, UniTensor, UniTensor, UniTensor, UniTensor]],
                 precision: str = "3xtf32", fp32: bool = True, tiles: Tuple[int, int] = (128, 64),
                 device: Optional[torch.device] = None):
        precision = precision.lower()
        if precision not in ("3xtf32", "bf16x3"):
            raise CytnxError("[BatchedTwoSiteHeff] precision must be '3xtf32' or 'bf16x3'")
        if not problems:
            raise CytnxError("[BatchedTwoSiteHeff] no problems")
        self.precision = precision
        self.prec = _lib.PRECISIONS[precision]
        self.fp32 = bool(fp32)
        self.dtype = torch.float32 if fp32 else torch.float64
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() \
                else torch.device("cpu")
        self.device = device
        self._plans: List[int] = []
        self._b = None
        self._graph = None
        # host planning of independent problems in parallel (the C++ planner runs with the GIL released)
        with ThreadPoolExecutor(max_workers=max(1, min(16, os.cpu_count() or 1))) as ex:
            futs = [ex.submit(plan_two_site, *prob, []) for prob in problems]
            results, err = [], None
            for f in futs:
                try:
                    results.append(f.result())
                except Exception as e:  # keep collecting so every created plan is destroyed
                    err = err or e
                    results.append(None)
        self._plans = [r[0] for r in results if r is not None]
        if err is not None:
            self._destroy_plans()
            raise err
        self.out_bonds = [r[2] for r in results]
        psi_n = [int(_lib.lib().ctn_heff2_psi_elems(r[0])) for r in results]
        L_n = [int(r[1][0]._layout.nelem) for r in results]
        R_n = [int(r[1][3]._layout.nelem) for r in results]
        self.nprob = len(self._plans)
        self.psi_sizes = np.array(psi_n, dtype=np.int64)
        self.L_sizes = np.array(L_n, dtype=np.int64)
        self.R_sizes = np.array(R_n, dtype=np.int64)
        self.psi_offsets, self.psi_total = _aligned_offsets(psi_n)
        self.L_offsets, self.L_total = _aligned_offsets(L_n)
        self.R_offsets, self.R_total = _aligned_offsets(R_n)
        self._ws = None
        self._env = None
        self._create(*tiles)

    # ---------------------------------------------------------------- lifetime
    def _destroy_plans(self):
        for h in self._plans:
            _lib.lib().ctn_heff2_plan_destroy(h)
        self._plans = []

    def _create(self, bn1: int, bn4: int) -> None:
        self._release_batch()
        arr = (ctypes.c_void_p * len(self._plans))(*self._plans)
        b = ctypes.c_void_p()
        P = _lib.P_i64
        _lib.check(_lib.lib().ctn_heff2_batch_create(arr, len(self._plans), self.psi_offsets.ctypes.data_as(P),
                                                     self.L_offsets.ctypes.data_as(P),
                                                     self.R_offsets.ctypes.data_as(P), self.prec, int(bn1), int(bn4),
                                                     1 if self.fp32 else 0, ctypes.byref(b)), "BatchedTwoSiteHeff")
        self._b = b.value
        self.tiles = (int(bn1), int(bn4))
        self._env = None

    def _release_batch(self):
        self._graph = None
        if self._b is not None:
            _lib.lib().ctn_heff2_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self._release_batch()
            self._destroy_plans()
        except Exception:
            pass

    # ---------------------------------------------------------------- accounting
    def workspace_bytes(self) -> int:
        return int(_lib.lib().ctn_heff2_batch_workspace_bytes(self._b))

    def gemm_flops(self) -> float:
        """Useful flops (2*M*N*K over every problem's stacked GEMM groups) of one batched matvec."""
        return float(_lib.lib().ctn_heff2_batch_gemm_flops(self._b))

    def gemm_stats(self) -> dict:
        """Work accounting of the two batched GEMMs (ctn_heff2_batch_stats): useful flops,
        executed MMA flops of the tiles (padding included, one product each) and the operand
        panel bytes the tiles copy into shared memory per matvec."""
        out = (ctypes.c_double * 8)()
        _lib.check(_lib.lib().ctn_heff2_batch_stats(self._b, out), "BatchedTwoSiteHeff.gemm_stats")
        return {f"step{s}": {"useful_flops": out[i], "executed_flops": out[i + 1], "panel_bytes": out[i + 2],
                             "operand_bytes": out[i + 3]} for s, i in ((1, 0), (4, 4))}

    def plan(self, i: int) -> int:
        return self._plans[i]

    # ---------------------------------------------------------------- flat buffers
    def gather(self, arrays: Sequence, which: str = "psi", pin: bool = False) -> torch.Tensor:
        """Concatenate per-problem flat data (numpy arrays or tensors) at the batch offsets
        into one device buffer of the batch dtype (``pin``: a pinned host buffer instead)."""
        offs, total, sizes = {"psi": (self.psi_offsets, self.psi_total, self.psi_sizes),
                              "L": (self.L_offsets, self.L_total, self.L_sizes),
                              "R": (self.R_offsets, self.R_total, self.R_sizes)}[which]
        if len(arrays) != self.nprob:
            raise CytnxError("[BatchedTwoSiteHeff.gather] one array per problem expected")
        host = torch.zeros(total, dtype=self.dtype, pin_memory=pin and torch.cuda.is_available())
        for i, a in enumerate(arrays):
            t = torch.as_tensor(a).reshape(-1)
            if t.numel() != sizes[i]:
                raise CytnxError(f"[BatchedTwoSiteHeff.gather] problem {i}: {t.numel()} elements, "
                                 f"expected {int(sizes[i])}")
            host[int(offs[i]): int(offs[i]) + t.numel()] = t.to(self.dtype).cpu()
        return host if pin else host.to(self.device)

    def slice(self, flat: torch.Tensor, i: int) -> torch.Tensor:
        """Problem i's part of a batch vector."""
        o = int(self.psi_offsets[i])
        return flat[o: o + int(self.psi_sizes[i])]

    # ---------------------------------------------------------------- binding and matvec
    def set_env(self, L_all: torch.Tensor, R_all: torch.Tensor) -> None:
        """Pack the environments of every problem (flat device buffers laid out by ``gather``)."""
        for t, nm, n in ((L_all, "L", self.L_total), (R_all, "R", self.R_total)):
            if t.dtype != self.dtype or t.numel() < n or not t.is_cuda:
                raise CytnxError(f"[BatchedTwoSiteHeff.set_env] {nm} must be a device {self.dtype} buffer of "
                                 f">= {n} elements")
        nbytes = self.workspace_bytes()
        if self._ws is None or self._ws.numel() < nbytes:
            self._ws = None
            self._ws = torch.empty(nbytes, dtype=torch.uint8, device=L_all.device)
        _lib.check(_lib.lib().ctn_heff2_batch_set_env(self._b, L_all.data_ptr(), R_all.data_ptr(), self._ws.data_ptr(),
                                                      _lib.stream_ptr()), "BatchedTwoSiteHeff.set_env")
        self._env = (L_all, R_all)
        self._graph = None

    def _check_vec(self, t: torch.Tensor, nm: str):
        if t.dtype != self.dtype or t.numel() < self.psi_total or not t.is_cuda:
            raise CytnxError(f"[BatchedTwoSiteHeff] {nm} must be a device {self.dtype} buffer of "
                             f">= {self.psi_total} elements")

    def matvec(self, psi_all: torch.Tensor, out_all: Optional[torch.Tensor] = None) -> torch.Tensor:
        """out = H_eff psi for every problem (one launch per phase).  Elements of out_all
        between the problems' slices are left untouched."""
        if self._env is None:
            raise CytnxError("[BatchedTwoSiteHeff] call set_env first")
        self._check_vec(psi_all, "psi")
        if out_all is None:
            out_all = torch.zeros_like(psi_all)
        self._check_vec(out_all, "out")
        _lib.check(_lib.lib().ctn_heff2_batch_matvec(self._b, psi_all.data_ptr(), out_all.data_ptr(),
                                                     _lib.stream_ptr()), "BatchedTwoSiteHeff.matvec")
        return out_all

    def profile(self, psi_all: torch.Tensor, out_all: torch.Tensor, reps: int = 5) -> List[float]:
        """Average per-phase times (ms): pack, step-1 GEMM, MPO fold, step-4 GEMM."""
        ms = (ctypes.c_double * 4)()
        _lib.check(_lib.lib().ctn_heff2_batch_profile(self._b, psi_all.data_ptr(), out_all.data_ptr(), int(reps), ms,
                                                      _lib.stream_ptr()), "BatchedTwoSiteHeff.profile")
        return [ms[i] for i in range(4)]

    # ---------------------------------------------------------------- CUDA graph
    def capture(self, psi_all: torch.Tensor, out_all: torch.Tensor) -> "torch.cuda.CUDAGraph":
        """Record one batched matvec on fixed buffers in a CUDA graph; ``replay`` runs it."""
        self.matvec(psi_all, out_all)  # first launch outside capture: kernel attributes, tables resident
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            _lib.check(_lib.lib().ctn_heff2_batch_matvec(self._b, psi_all.data_ptr(), out_all.data_ptr(),
                                                         _lib.stream_ptr()), "BatchedTwoSiteHeff.capture")
        self._graph = (g, psi_all, out_all)
        return g

    def replay(self) -> torch.Tensor:
        if self._graph is None:
            raise CytnxError("[BatchedTwoSiteHeff] nothing captured")
        self._graph[0].replay()
        return self._graph[2]

    # ---------------------------------------------------------------- tile autotuner
    def autotune(self, psi_all: torch.Tensor, step1=(64, 96, 128, 160, 192), step4=(32, 48, 64, 96, 128),
                 reps: int = 5) -> Dict:
        """Pick the tile widths of the two batched GEMMs by timing: each phase is its own
        kernel, so step 1 is tuned with step 4 fixed, then step 4 with the best step 1.
        Every candidate rebuilds the batch tables and re-packs the environments."""
        if self._env is None:
            raise CytnxError("[BatchedTwoSiteHeff.autotune] call set_env first")
        L_all, R_all = self._env
        out = torch.zeros_like(psi_all)

        def phase_ms(b1, b4):
            self._create(b1, b4)
            self.set_env(L_all, R_all)
            self.matvec(psi_all, out)
            return self.profile(psi_all, out, reps)

        fixed4 = self.tiles[1]
        t1 = {b: phase_ms(b, fixed4)[1] for b in step1}
        best1 = min(t1, key=t1.get)
        t4 = {b: phase_ms(best1, b)[3] for b in step4}
        best4 = min(t4, key=t4.get)
        self._create(best1, best4)
        self.set_env(L_all, R_all)
        return {"step1": best1, "step4": best4, "ms_step1": t1, "ms_step4": t4}


def problem_flops(problem) -> float:
    """Algorithmic flops of one matvec of a structure-only two-site problem (L, M1, M2, R,
    psi): 2*m*n*k over every block pair of the four contractions L -> M1 -> M2 -> R, counted
    on the host (the cost model of the sharding)."""
    from .heff import _struct_contract
    from .unitensor import contract_plan_flops, structure_only

    L, M1, M2, R, psi = problem
    P = structure_only(psi.bonds(), ["a", "s1", "s2", "b"])
    Ls = structure_only(L.bonds(), ["w", "a", "ap"])
    M1s = structure_only(M1.bonds(), ["w", "w1", "s1", "s1p"])
    M2s = structure_only(M2.bonds(), ["w1", "w2", "s2", "s2p"])
    Rs = structure_only(R.bonds(), ["w2", "b", "bp"])
    f = contract_plan_flops(Ls, P)
    T = _struct_contract(Ls, P)
    for X in (M1s, M2s, Rs):
        f += contract_plan_flops(T, X)
        T = _struct_contract(T, X)
    return f


def shard_problems(costs: Sequence[float], nshards: int) -> List[List[int]]:
    """Split problems over ``nshards`` ranks by longest-processing-time-first: problems in
    decreasing cost go to the currently lightest shard (ties: lowest rank).  Deterministic,
    so every rank computes the same assignment without communicating."""
    if nshards < 1:
        raise CytnxError("[shard_problems] nshards must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * nshards
    shards: List[List[int]] = [[] for _ in range(nshards)]
    for i in order:
        r = min(range(nshards), key=lambda k: (load[k], k))
        shards[r].append(i)
        load[r] += float(costs[i])
    return [sorted(s) for s in shards]
