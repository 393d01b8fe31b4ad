"""linalg.Lanczos_Exp (exp(tau H) v by Lanczos projection; src/linalg/Lanczos_Exp.cpp) against
the matrix exponential of the dense operator (scipy.linalg.expm), for a Tensor operator, a
dense UniTensor network operator and the planned block-sparse two-site H_eff."""
import numpy as np
import pytest
import scipy.linalg
import torch

pytestmark = pytest.mark.gpu


def _sym(n, seed, scale=1.0):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((n, n))
    return scale * (A + A.T) / (2 * np.sqrt(n)), rng


@pytest.mark.parametrize("tau", [-0.5, -2.0, 0.3, -0.7j, 0.2 - 0.4j])
def test_tensor_operator_matches_expm(tau):
    import cytnx_b200 as c

    n = 200
    A, rng = _sym(n, 11, scale=3.0)
    At = torch.from_numpy(A).cuda()

    class Op(c.LinOp):
        def matvec(self, v):
            return c.Tensor.from_torch(At @ v.to_torch())

    v = rng.standard_normal(n)
    out = c.linalg.Lanczos_Exp(Op("mv", n), c.Tensor.from_torch(torch.from_numpy(v).cuda()), tau, CvgCrit=1e-14)
    got = out.to_torch().cpu().numpy()
    ref = scipy.linalg.expm(tau * A) @ v
    assert got.dtype == (np.float64 if complex(tau).imag == 0 else np.complex128)
    assert np.linalg.norm(got - ref) <= 1e-11 * np.linalg.norm(ref)


def test_invariant_subspace_breakdown():
    """v in the span of three eigenvectors: the recurrence stops at dimension 3 (beta below
    the breakdown bound) and the result is exact."""
    import cytnx_b200 as c

    n = 120
    A, rng = _sym(n, 5)
    w, Q = np.linalg.eigh(A)
    v = Q[:, [3, 50, 100]] @ np.array([0.3, -1.2, 0.8])
    At = torch.from_numpy(A).cuda()

    class Op(c.LinOp):
        def matvec(self, x):
            return c.Tensor.from_torch(At @ x.to_torch())

    out = c.linalg.Lanczos_Exp(Op("mv", n), c.Tensor.from_torch(torch.from_numpy(v).cuda()), -1.0, CvgCrit=1e-300,
                               Maxiter=50)
    ref = scipy.linalg.expm(-1.0 * A) @ v
    assert np.linalg.norm(out.to_torch().cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)


def test_block_two_site_heff_matches_expm():
    """The planned block-sparse H_eff (FP64) as the LinOp on a block UniTensor."""
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    psi, L, M1, M2, R = W.build_two_site(W.xxz_spec(16), W.xxz_mpo_values(1.0, 1.0), seed=4, device=0)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    x = psi.flat_view()
    n = x.numel()
    Hd = np.zeros((n, n))
    e = torch.zeros_like(x)
    y = torch.empty_like(x)
    for i in range(n):
        e.zero_()
        e[i] = 1.0
        H.apply_flat(e, y, "fp64")
        Hd[:, i] = y.cpu().numpy()
    Hd = 0.5 * (Hd + Hd.T)
    tau = -0.05
    out = c.linalg.Lanczos_Exp(H, psi, tau, CvgCrit=1e-14)
    assert out.labels() == psi.labels()
    got = out.flat_view().cpu().numpy()
    ref = scipy.linalg.expm(tau * Hd) @ x.cpu().numpy()
    assert np.linalg.norm(got - ref) <= 1e-10 * np.linalg.norm(ref)
