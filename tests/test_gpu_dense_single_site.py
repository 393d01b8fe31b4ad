"""Plain dense FP64 single-site DMRG matvec (the CPU-runnable configuration):
L[64,5,64] and R[64,5,64] ~N(0,1) symmetrised over their two bond indices, the exact
spin-1/2 XXZ MPO W[5,5,2,2] (Jz = Jxy = 1, h = 0), A[64,2,64] ~N(0,1) normalised;
30 Lanczos iterations for the ground state through Network / LinOp / linalg.Lanczos,
against the oracle (numpy einsum matvec + the oracle's Lanczos_Gnd_Ut restatement)."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def _operands(seed=0, D=64):
    from cytnx_b200 import workloads as W

    rng = np.random.default_rng(seed)
    L = rng.standard_normal((D, 5, D))
    L = 0.5 * (L + L.transpose(2, 1, 0))
    R = rng.standard_normal((D, 5, D))
    R = 0.5 * (R + R.transpose(2, 1, 0))
    Wm = np.zeros((5, 5, 2, 2))
    for (a, b, s, sp), v in W.xxz_mpo_values(1.0, 1.0, 0.0).items():
        Wm[a, b, s, sp] = v
    A = rng.standard_normal((D, 2, D))
    A /= np.linalg.norm(A)
    return L, Wm, R, A


def _oracle_matvec(L, Wm, R):
    def mv(x):
        A = x.reshape(L.shape[0], 2, R.shape[0])
        # out[a', s', b'] = sum L[a,w,a'] A[a,s,b] W[w,w2,s,s'] R[b,w2,b']
        t = np.einsum("awx,asb->wxsb", L, A)
        t = np.einsum("wxsb,wvsy->xyvb", t, Wm)
        return np.einsum("xyvb,bvz->xyz", t, R).reshape(-1)
    return mv


def test_dense_single_site_lanczos_30_iterations():
    import cytnx_b200 as c

    L, Wm, R, A = _operands()
    dev = torch.device("cuda", 0)
    Lu = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(L).to(dev)), False, -1, ["a", "w", "ap"])
    Ru = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(R).to(dev)), False, -1, ["b", "w2", "bp"])
    Wu = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(Wm).to(dev)), False, -1, ["w", "w2", "s", "sp"])
    Au = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(A).to(dev)), False, -1, ["a", "s", "b"])

    class OneSite(c.LinOp):
        def __init__(self):
            super().__init__("mv", A.size, c.Type.Double, c.Device.cuda)
            self.net = c.Network()
            self.net.FromString(["A: a,s,b", "L: a,w,ap", "W: w,w2,s,sp", "R: b,w2,bp", "TOUT: ap,sp,bp"])
            self.net.PutUniTensors(["L", "W", "R"], [Lu, Wu, Ru])

        def matvec(self, v):
            lbl = v.labels()
            self.net.PutUniTensor("A", v)
            out = self.net.Launch()
            out.relabel_(lbl)
            return out

    H = OneSite()
    mv = _oracle_matvec(L, Wm, R)
    # one matvec against the oracle
    y = H.matvec(Au).get_block_().to_torch().cpu().numpy().reshape(-1)
    ref = mv(A.reshape(-1))
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) < 1e-13
    # 30 Lanczos iterations, the reference's recurrence on both sides
    E, vec = c.linalg.Lanczos(Hop=H, Tin=Au, method="Gnd", Maxiter=30, CvgCrit=1e-300)
    E_ref, v_ref, it = O.lanczos_gnd_ut(mv, A.reshape(-1), 1e-300, 30)
    assert it == 30
    e = float(E.item()) if hasattr(E, "item") else float(E)
    assert abs(e - E_ref) / abs(E_ref) < 1e-10
    # the returned vector is the reference's combination sum_n kry[n] psi_s[n] of the stored
    # Krylov vectors; run 30 iterations past convergence it is not a unit vector (the
    # unreorthogonalised recurrence has ghost copies of the converged eigenvalue), and the
    # same combination is reproduced here (eigenvector sign is arbitrary)
    v = vec.get_block_().to_torch().cpu().numpy().reshape(-1)
    d = min(np.linalg.norm(v - v_ref), np.linalg.norm(v + v_ref)) / np.linalg.norm(v_ref)
    assert d < 1e-6, d
