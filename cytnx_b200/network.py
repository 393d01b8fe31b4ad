"""Network (text-defined contraction of several UniTensors) and LinOp.

Network mirrors ``cytnx::Network`` / ``RegularNetwork`` (src/RegularNetwork.cpp:901-1007):
``FromString`` lines ``"name: l1,l2;l3"``, ``"TOUT: a,b;c"``, optional ``"ORDER: ((A,B),C)"``;
``PutUniTensor`` (relabel to the network labels), ``Launch`` = post-order walk of a
binary contraction tree, default tree = left fold in declaration order
(src/contraction_tree.cpp:6-30), ORDER tokens (:32-124), ``setOrder(optimal=True)``
= cost-based search over pairwise orders.  Every pairwise step is the planned
block-sparse contract (plans cached across Launch calls).

LinOp mirrors ``cytnx::LinOp`` (include/LinOp.hpp:68-167): subclass and override
``matvec``.
"""
from __future__ import annotations

import itertools
import re
from typing import Dict, List, Optional, Sequence

import numpy as np

from ._lib import CytnxError
from .core import Device, Type
from .unitensor import Contract, UniTensor


def _split_labels(s: str) -> List[str]:
    s = s.strip()
    if not s:
        return []
    return [x.strip().strip("'\"") for x in s.split(",") if x.strip()]


class Network:
    def __init__(self, fname: Optional[str] = None):
        self._names: List[str] = []
        self._labels: List[List[str]] = []
        self._tensors: Dict[str, UniTensor] = {}
        self._tout: List[str] = []
        self._tout_rowrank = 0
        self._order: Optional[str] = None
        self._optimal = False
        if fname:
            self.Fromfile(fname)

    # -------------------------------------------------------------- definition
    def Fromfile(self, fname: str) -> None:
        with open(fname) as f:
            self.FromString([l for l in f.read().splitlines() if l.strip() and not l.strip().startswith("#")])

    def FromString(self, contents: Sequence[str]) -> None:
        self.__init__()
        for line in contents:
            line = line.split("#")[0].strip()
            if not line:
                continue
            if ":" not in line:
                raise CytnxError(f"[ERROR][Network] invalid line '{line}'")
            name, rest = line.split(":", 1)
            name = name.strip()
            if name == "TOUT":
                if ";" in rest:
                    a, b = rest.split(";", 1)
                    la, lb = _split_labels(a), _split_labels(b)
                else:
                    la, lb = _split_labels(rest), []
                self._tout = la + lb
                self._tout_rowrank = len(la)
            elif name == "ORDER":
                self._order = rest.strip()
            else:
                if name in self._names:
                    raise CytnxError(f"[ERROR][Network] duplicated tensor name '{name}'")
                labs = _split_labels(rest.replace(";", ","))
                self._names.append(name)
                self._labels.append(labs)
        if len(self._names) < 1:
            raise CytnxError("[ERROR][Network] no tensor declared")

    def PutUniTensor(self, name, utensor: UniTensor, label_order: Sequence[str] = ()) -> None:
        if isinstance(name, int):
            name = self._names[name]
        if name not in self._names:
            raise CytnxError(f"[ERROR][Network] no tensor named '{name}'")
        if label_order:
            utensor = utensor.permute(list(label_order))
        labs = self._labels[self._names.index(name)]
        if utensor.rank() != len(labs):
            raise CytnxError(f"[ERROR][Network] tensor '{name}' rank {utensor.rank()} != {len(labs)} labels")
        self._tensors[name] = utensor.relabel(labs)

    def PutUniTensors(self, names: Sequence[str], utensors: Sequence[UniTensor]) -> None:
        for n, u in zip(names, utensors):
            self.PutUniTensor(n, u)

    def RmUniTensor(self, name) -> None:
        if isinstance(name, int):
            name = self._names[name]
        self._tensors.pop(name, None)

    def setOrder(self, optimal: bool = False, contract_order: str = "") -> None:
        self._optimal = bool(optimal)
        if contract_order:
            self._order = contract_order

    def getOrder(self) -> str:
        return self._order or self._default_order_str()

    def _default_order_str(self) -> str:
        s = self._names[0]
        for n in self._names[1:]:
            s = f"({s},{n})"
        return s

    # -------------------------------------------------------------- trees
    def _parse_order(self, s: str):
        toks = re.findall(r"\(|\)|,|[^(),\s]+", s)
        pos = 0

        def expr():
            nonlocal pos
            t = toks[pos]
            if t == "(":
                pos += 1
                items = [expr()]
                while toks[pos] == ",":
                    pos += 1
                    items.append(expr())
                if toks[pos] != ")":
                    raise CytnxError("[ERROR][Network] malformed ORDER")
                pos += 1
                node = items[0]
                for it in items[1:]:
                    node = (node, it)
                return node
            pos += 1
            if t not in self._names:
                raise CytnxError(f"[ERROR][Network] ORDER names unknown tensor '{t}'")
            return t

        tree = expr()
        return tree

    def _cost_tree(self) -> tuple:
        """Cheapest pairwise order by exhaustive search on dense-equivalent flop counts
        (the role of getOptimalOrder / SearchTree, src/search_tree.cpp:9-150)."""
        dims: Dict[str, int] = {}
        for n in self._names:
            u = self._tensors[n]
            for l, d in zip(u.labels(), u.shape()):
                dims[l] = d
        best = {}
        items = {frozenset([n]): (0.0, n, frozenset(self._tensors[n].labels())) for n in self._names}
        best.update(items)
        names = list(self._names)
        allset = frozenset(names)
        for size in range(2, len(names) + 1):
            for combo in itertools.combinations(names, size):
                S = frozenset(combo)
                cand = None
                lst = list(S)
                for r in range(1, size // 2 + 1):
                    for left in itertools.combinations(lst, r):
                        L = frozenset(left)
                        R = S - L
                        if L not in best or R not in best:
                            continue
                        cl, tl, ll = best[L]
                        cr, tr, lr = best[R]
                        comm = ll & lr
                        outl = ll ^ lr
                        cost = float(np.prod([dims[x] for x in ll | lr])) if (ll | lr) else 1.0
                        tot = cl + cr + cost
                        if cand is None or tot < cand[0]:
                            cand = (tot, (tl, tr), frozenset(outl))
                if cand is not None:
                    best[S] = cand
        return best[allset][1]

    # -------------------------------------------------------------- launch
    def Launch(self) -> UniTensor:
        missing = [n for n in self._names if n not in self._tensors]
        if missing:
            raise CytnxError(f"[ERROR][Network] tensors not set: {missing}")
        if len(self._names) == 1:
            out = self._tensors[self._names[0]]
        else:
            if self._order:
                tree = self._parse_order(self._order)
            elif self._optimal:
                tree = self._cost_tree()
            else:
                tree = self._names[0]
                for n in self._names[1:]:
                    tree = (tree, n)
            out = self._eval(tree)
        if self._tout:
            if sorted(out.labels()) != sorted(self._tout):
                raise CytnxError(f"[ERROR][Network] TOUT labels {self._tout} do not match result {out.labels()}")
            out = out.permute(self._tout, self._tout_rowrank)
        return out

    def _eval(self, node) -> UniTensor:
        if isinstance(node, str):
            return self._tensors[node]
        a = self._eval(node[0])
        b = self._eval(node[1])
        return Contract(a, b)

    def clear(self) -> None:
        self._tensors.clear()

    def __repr__(self):
        lines = [f"{n}: {','.join(l)}" for n, l in zip(self._names, self._labels)]
        lines.append("TOUT: " + ",".join(self._tout[: self._tout_rowrank]) + ";" + ",".join(self._tout[self._tout_rowrank:]))
        return "Network(\n  " + "\n  ".join(lines) + "\n)"


class LinOp:
    """User operator: subclass and override ``matvec(v)`` (include/LinOp.hpp:68-167)."""

    def __init__(self, type: str = "mv", nx: int = 0, dtype: int = Type.Double, device: int = Device.cuda):
        if type not in ("mv", "mv_elem"):
            raise CytnxError("[ERROR][LinOp] type must be 'mv' or 'mv_elem'")
        self._type = type
        self._nx = int(nx)
        self._dtype = dtype
        self._device = device

    def nx(self) -> int:
        return self._nx

    def dtype(self) -> int:
        return self._dtype

    def device(self) -> int:
        return self._device

    def matvec(self, v):
        raise CytnxError("[ERROR][LinOp] matvec is not overridden")
