"""A two-site U(1) DMRG driver written against the cytnx Python API.

It exercises the calls the reference's DMRG example scripts make
(example/DMRG/dmrg_two_sites_U1.py): Bond/UniTensor construction with U(1) quantum
numbers, set_elem, Contract, Network.FromString/PutUniTensors/Launch with TOUT, a
LinOp subclass driven by linalg.Lanczos(method="Gnd"), Dagger().permute_(...),
linalg.Svd_truncate, relabel_ and scalar arithmetic.  The module under test is passed
in (``cytnx_b200``), so the same driver runs unchanged against any implementation of
that API.  ``planned=True`` swaps the Network-based LinOp for the planned two-site
operator (TwoSiteHeff), which must give the same energies.
"""
import numpy as np

from cytnx_b200 import workloads as W


def _env_left(c, Lenv, A, M):
    """L'[w', b, b'] = sum L[w,a,a'] A[a,s,b] M[w,w',s,s'] A*[a',s',b']."""
    net = c.Network()
    net.FromString(["L: w,a,ap", "A: a,s,b", "M: w,wn,s,sp", "Ac: ap,sp,bp", "TOUT: wn;b,bp"])
    Ad = A.Dagger().permute_(A.labels())
    net.PutUniTensors(["L", "A", "M", "Ac"], [Lenv, A, M, Ad])
    return net.Launch()


def _env_right(c, Renv, A, M):
    """R'[w, a, a'] = sum A[a,s,b] R[w',b,b'] M[w,w',s,s'] A*[a',s',b']."""
    net = c.Network()
    net.FromString(["R: wn,b,bp", "A: a,s,b", "M: w,wn,s,sp", "Ac: ap,sp,bp", "TOUT: w;a,ap"])
    Ad = A.Dagger().permute_(A.labels())
    net.PutUniTensors(["R", "A", "M", "Ac"], [Renv, A, M, Ad])
    return net.Launch()


def _make_linop(c, Lenv, M, Renv, psi):
    class TwoSiteOp(c.LinOp):
        def __init__(self):
            super().__init__("mv", int(np.prod(psi.shape())), c.Type.Double, c.Device.cuda)
            self.net = c.Network()
            self.net.FromString(["psi: a,s1,s2,b", "L: w,a,ap", "R: w2,b,bp", "M1: w,w1,s1,s1p",
                                 "M2: w1,w2,s2,s2p", "TOUT: ap,s1p;s2p,bp"])
            self.net.PutUniTensors(["L", "M1", "M2", "R"], [Lenv, M, M, Renv])

        def matvec(self, v):
            lbl = v.labels()
            self.net.PutUniTensor("psi", v)
            out = self.net.Launch()
            out.relabel_(lbl)
            return out

    return TwoSiteOp()


def run(c, nsites=20, chi=32, sweeps=6, lanczos_maxiter=4, cvgcrit=1e-12, Jz=0.0, Jxy=2.0, planned=False):
    M, inner, phys = W.xxz_mpo_unitensor(Jz, Jxy, device=0)
    v0 = c.Bond(c.BD_KET, [[0]], [1])
    Lb = c.UniTensor([inner.redirect(), v0.redirect(), v0], labels=["w", "a", "ap"], rowrank=1, device=0)
    Lb.set_elem([0, 0, 0], 1.0)          # left boundary: MPO channel 0
    Rb = c.UniTensor([inner, v0, v0.redirect()], labels=["w", "b", "bp"], rowrank=1, device=0)
    Rb.set_elem([4, 0, 0], 1.0)          # right boundary: MPO channel 4
    # Neel product state with the total charge returning to 0
    A, left, q = [], v0, 0
    for k in range(nsites):
        s = k % 2
        q_right = q - int(phys._qnums[s][0])
        right = c.Bond(c.BD_BRA, [[q_right]], [1])
        t = c.UniTensor([left, phys.redirect(), right], labels=[f"v{k}", f"p{k}", f"v{k + 1}"], rowrank=2, device=0)
        t.set_elem([0, s, 0], 1.0)
        A.append(t)
        left, q = right.redirect(), q_right
    labels = [[f"v{k}", f"p{k}", f"v{k + 1}"] for k in range(nsites)]

    L = [None] * (nsites + 1)
    R = [None] * (nsites + 1)
    L[0] = Lb
    R[nsites] = Rb
    for k in range(nsites - 1):
        L[k + 1] = _env_left(c, L[k], A[k].relabel(["a", "s", "b"]), M.relabel(["w", "wn", "s", "sp"]))
    energies = []

    def optimize(p):
        psi = c.Contract(A[p], A[p + 1]).relabel(["a", "s1", "s2", "b"])
        if planned:
            H = c.TwoSiteHeff(L[p], M, M, R[p + 2], psi)
        else:
            H = _make_linop(c, L[p], M, R[p + 2], psi)
        E, vec = c.linalg.Lanczos(Hop=H, method="Gnd", Maxiter=lanczos_maxiter, CvgCrit=cvgcrit, Tin=psi)
        energies.append(E.item())
        vec.set_rowrank_(2)
        dl, dr = A[p].shape()[0], A[p + 1].shape()[2]
        return c.linalg.Svd_truncate(vec, min(dl * 2, dr * 2, chi))

    for sweep in range(sweeps):
        for p in range(nsites - 2, -1, -1):  # right to left
            S, U, Vt = optimize(p)
            S = S / S.norm()
            A[p + 1] = Vt.relabel(labels[p + 1])
            A[p] = c.Contract(U, S).relabel(labels[p])
            R[p + 1] = _env_right(c, R[p + 2], A[p + 1].relabel(["a", "s", "b"]), M.relabel(["w", "wn", "s", "sp"]))
        for p in range(nsites - 1):  # left to right
            S, U, Vt = optimize(p)
            S = S / S.norm()
            A[p] = U.relabel(labels[p])
            A[p + 1] = c.Contract(S, Vt).relabel(labels[p + 1])
            L[p + 1] = _env_left(c, L[p], A[p].relabel(["a", "s", "b"]), M.relabel(["w", "wn", "s", "sp"]))
    return energies


def free_fermion_energy(nsites, Jxy=2.0):
    """XX chain H = (Jxy/2) sum (S+S- + S-S+): Jordan-Wigner free fermions with hopping Jxy/2."""
    h = np.diag(np.ones(nsites - 1), 1) + np.diag(np.ones(nsites - 1), -1)
    e = np.linalg.eigvalsh(h) * (Jxy / 2.0)
    return float(e[e < 0].sum())
