"""The which form of linalg.Lanczos (k extreme eigenpairs; ARPACK in the reference,
src/linalg/Lanczos.cpp:250-580) against exact diagonalisation, as the reference's LanczosUt
tests do (tests/linalg_test/Lanczos_Gnd_test.cpp:203-310: eigenvalues vs Eigh to 1e-12,
residual |Hv - ev| < 1e-12, k up to dim - 2, is_V false)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _one_site_op(D=5, d=2, dw=3, seed=0):
    """One-site effective Hamiltonian as in the reference test: L[D,dw,D], O[dw,d,dw,d],
    R[D,dw,D] ~ U(-1, 1) made Hermitian, contracted by a Network inside LinOp.matvec."""
    import cytnx_b200 as c

    rng = np.random.default_rng(seed)
    L = rng.uniform(-1, 1, (D, dw, D))
    L = L + L.transpose(2, 1, 0)
    R = rng.uniform(-1, 1, (D, dw, D))
    R = R + R.transpose(2, 1, 0)
    O = rng.uniform(-1, 1, (dw, d, dw, d))
    O = O + O.transpose(0, 3, 2, 1)
    dev = torch.device("cuda", 0)
    Lu = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(L).to(dev)), False, -1, ["vil", "Lm", "vol"])
    Ru = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(R).to(dev)), False, -1, ["vir", "Rm", "vor"])
    Ou = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(O).to(dev)), False, -1, ["Lm", "pi", "Rm", "po"])
    # dense H[(vol po vor), (vil pi vir)] for the exact spectrum
    Hd = np.einsum("amx,mpnq,bny->xqyapb", L, O, R).reshape(D * d * D, D * d * D)
    psi0 = rng.uniform(-1, 1, (D, d, D))

    class OneSite(c.LinOp):
        def __init__(self):
            super().__init__("mv", D * d * D, c.Type.Double, c.Device.cuda)
            self.net = c.Network()
            self.net.FromString(["psi: vil, pi, vir", "L: vil, Lm, vol", "O: Lm, pi, Rm, po", "R: vir, Rm, vor",
                                 "TOUT: vol, po, vor"])
            self.net.PutUniTensors(["L", "O", "R"], [Lu, Ou, Ru])

        def matvec(self, v):
            lbl = v.labels()
            self.net.PutUniTensor("psi", v)
            out = self.net.Launch()
            out.relabel_(lbl)
            return out

    Tin = c.UniTensor(c.Tensor.from_torch(torch.from_numpy(psi0).to(dev)), False, -1, ["vil", "pi", "vir"])
    return OneSite(), Tin, Hd


def _order(ev, which, k):
    if which == "SA":
        return np.sort(ev)[:k]
    if which == "LA":
        return np.sort(ev)[::-1][:k]
    return ev[np.argsort(-np.abs(ev), kind="stable")][:k]


def test_dense_one_site_operator_is_symmetric():
    _, _, Hd = _one_site_op()
    assert np.abs(Hd - Hd.T).max() < 1e-12


@pytest.mark.parametrize("which", ["SA", "LA", "LM"])
@pytest.mark.parametrize("k", [1, 3])
def test_which_matches_exact_spectrum(which, k):
    import cytnx_b200 as c

    H, Tin, Hd = _one_site_op()
    out = c.linalg.Lanczos(H, Tin, which=which, k=k, Maxiter=10000, CvgCrit=0)
    assert len(out) == k + 1
    ev = out[0].get_block_().numpy()
    ref = _order(np.linalg.eigvalsh(Hd), which, k)
    assert ev.shape == (k,)
    assert np.all(np.abs(np.abs(ev) - np.abs(ref)) <= 1e-12 * np.abs(ref)), (ev, ref)
    for i in range(k):
        v = out[i + 1]
        assert v.labels() == Tin.labels()
        x = v.get_block_().numpy().reshape(-1)
        assert abs(np.linalg.norm(x) - 1.0) < 1e-12
        assert np.linalg.norm(Hd @ x - ev[i] * x) < 1e-12 * max(1.0, abs(ev[i]))


def test_k_close_to_dimension_and_no_vectors():
    """k = dim - 2 (the reference's KLarge case), and is_V = False returns the same values."""
    import cytnx_b200 as c

    H, Tin, Hd = _one_site_op(D=3, d=2, dw=2, seed=3)  # dim 18
    k = 16
    out = c.linalg.Lanczos(H, Tin, which="LM", k=k, CvgCrit=0)
    ev = out[0].get_block_().numpy()
    ref = _order(np.linalg.eigvalsh(Hd), "LM", k)
    assert np.all(np.abs(np.abs(ev) - np.abs(ref)) <= 1e-12 * np.abs(ref))
    noV = c.linalg.Lanczos(H, Tin, which="LM", k=k, CvgCrit=0, is_V=False)
    assert len(noV) == 1 and len(out) == k + 1
    assert np.abs(noV[0].get_block_().numpy() - ev).max() < 1e-12 * np.abs(ev).max()


def test_tensor_operator_restarts():
    """A 400-dimensional Tensor operator with clustered low eigenvalues: k = 6 lowest with a
    small basis (ncv = 16), so the thick restart has to run many cycles."""
    import cytnx_b200 as c

    n = 400
    rng = np.random.default_rng(7)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    lam = np.concatenate([np.linspace(-3.0, -2.9, 6), rng.uniform(-1.0, 5.0, n - 6)])
    A = (Q * lam) @ Q.T
    A = 0.5 * (A + A.T)
    At = torch.from_numpy(A).cuda()

    class Op(c.LinOp):
        def matvec(self, v):
            return c.Tensor.from_torch(At @ v.to_torch())

    x0 = c.Tensor.from_torch(torch.from_numpy(rng.standard_normal(n)).cuda())
    ev, vec = c.linalg.Lanczos(Op("mv", n), x0, which="SA", k=6, ncv=16, CvgCrit=1e-13)
    e = ev.numpy()
    ref = np.sort(np.linalg.eigvalsh(A))[:6]
    assert np.abs(e - ref).max() < 1e-11
    V = vec.numpy()
    assert V.shape == (6, n)
    for i in range(6):
        assert np.linalg.norm(A @ V[i] - e[i] * V[i]) < 1e-10
