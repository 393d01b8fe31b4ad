"""Environment updates of a DMRG sweep.

The left and right environment recursions of example/DMRG/dmrg_two_sites_U1.py
(:115-126 and :191-200 for the left update L' = L A M A^dagger, :151-161 for the right
update R' = A R M A^dagger), which the example runs as four-tensor Networks:

    left:   L'[b, wn, bp] = sum L[w, a, ap] A[a, s, b] M[w, wn, s, sp] A*[ap, sp, bp]
    right:  R'[w, a, ap]  = sum A[a, s, b] R[wn, b, bp] M[w, wn, s, sp] A*[ap, sp, bp]

Each update is three pairwise block-sparse contractions in a fixed order (the order the
example's networks contract by default): env . A, then . M, then . A^dagger, every one a
planned grouped FP64 GEMM on the device (ctn_contract_plan_*; plans are built once per
block structure and reused for every site and sweep with the same bonds).  The result is
returned with the input environment's leg order and labels, so it can feed the next
update and the two-site H_eff directly.
"""
from __future__ import annotations

from .unitensor import Contract, UniTensor

_ENV = ["w", "a", "ap"]


def _dagger(A: UniTensor, labels) -> UniTensor:
    """A^dagger with A's legs relabelled (real data: the bonds are redirected, values unchanged)."""
    return A.Dagger().relabel(list(reversed(labels)))


def left_update(L: UniTensor, A: UniTensor, M: UniTensor) -> UniTensor:
    """L'[w, a, ap] from L[w, a, ap] (legs w: MPO, a: ket bond, ap: bra bond), the site tensor
    A[a, s, b] (legs in that order: left bond, physical, right bond) and the MPO
    M[w, wn, s, sp].  Labels of the inputs are not used (the legs are taken by position)."""
    Lr = L.relabel(_ENV)
    Ar = A.relabel(["a", "s", "b"])
    Mr = M.relabel(["w", "wn", "s", "sp"])
    t = Contract(Lr, Ar)                       # (w, ap, s, b)
    t = Contract(t, Mr)                        # (ap, b, wn, sp)
    t = Contract(t, _dagger(Ar, ["ap", "sp", "bp"]))  # (b, wn, bp)
    t = t.relabel([{"b": "a", "wn": "w", "bp": "ap"}[l] for l in t.labels()])
    return t.permute(_ENV, 1).relabel(L.labels())


def right_update(R: UniTensor, A: UniTensor, M: UniTensor) -> UniTensor:
    """R'[w, a, ap] from R[w, b, bp], the site tensor A[a, s, b] and the MPO M[w, wn, s, sp]
    (legs by position; the result has R's leg order and labels)."""
    Rr = R.relabel(["wn", "b", "bp"])
    Ar = A.relabel(["a", "s", "b"])
    Mr = M.relabel(["w", "wn", "s", "sp"])
    t = Contract(Ar, Rr)                       # (a, s, wn, bp)
    t = Contract(t, Mr)                        # (a, bp, w, sp)
    t = Contract(t, _dagger(Ar, ["ap", "sp", "bp"]))  # (a, w, ap)
    return t.permute(_ENV, 1).relabel(R.labels())
