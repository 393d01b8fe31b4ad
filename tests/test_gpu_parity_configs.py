"""The CUDA path against the oracle at the benchmark configurations' own sizes.

Inputs: the oracle builds its operators with its own generator (oracle/workloads.py) and
the product with cytnx_b200.workloads; a CPU test pins the two to identical values.

* config 2 (U(1) XXZ, D=1024, FP64): one matvec, and 40 iterations of the reference's
  Lanczos_Gnd_Ut recurrence against ``oracle.lanczos_gnd_ut`` driven by the oracle matvec.
* config 3 (D=4096): the FP64 matvec, the split-precision matvecs' errors, and the
  refined ground state checked with the oracle's own FP64 matvec (its Rayleigh quotient
  and eigen-residual of the returned vector).
* config 5: the gradient of <A|H|A> equals 2 H_eff A_k with H_eff built by the oracle's
  contractions (environments included).
"""
import numpy as np
import pytest
import torch

import oracle as O
from oracle import workloads as OW

pytestmark = pytest.mark.gpu


def _product(D, seed=0):
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    psi, L, M1, M2, R = W.build_two_site(W.xxz_spec(D), W.xxz_mpo_values(), seed=seed, device=0)
    return c.TwoSiteHeff(L, M1, M2, R, psi), psi


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def cfg2():
    O.set_threads(__import__("os").cpu_count() or 1)
    H, psi = _product(1024)
    return H, psi, OW.xxz_two_site(1024, seed=0)


def test_config2_matvec_matches_oracle(cfg2):
    H, psi, ops = cfg2
    got = H.matvec(psi).flat_view().cpu().numpy()
    ref = OW.heff_matvec(ops)
    assert _rel(got, ref) <= 1e-12


def test_config2_lanczos_40_iterations_matches_oracle(cfg2):
    """Lanczos_Gnd_Ut.cpp:29-162, 40 iterations (no early stop): same iteration count,
    energies to 1e-10 relative, Ritz vectors to 1e-6."""
    H, psi, ops = cfg2
    E, vec, it = H.lanczos(psi, maxiter=40, cvgcrit=1e-300)
    x0 = ops["psi"].flat()
    E_ref, v_ref, it_ref = O.lanczos_gnd_ut(lambda x: OW.heff_matvec(ops, x), x0, 1e-300, 40)
    assert it == it_ref == 40
    assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
    v = vec.flat_view().cpu().numpy()
    assert min(np.linalg.norm(v - v_ref), np.linalg.norm(v + v_ref)) <= 1e-6 * np.linalg.norm(v_ref)


@pytest.fixture(scope="module")
def cfg3():
    O.set_threads(__import__("os").cpu_count() or 1)
    H, psi = _product(4096)
    ops = OW.xxz_two_site(4096, seed=0)
    return H, psi, ops, OW.heff_matvec(ops)


def test_config3_matvecs_against_oracle(cfg3):
    """FP64 form to 1e-12; the split forms' matvec errors against the oracle's FP64
    matvec stay at their representation / FP32-accumulation level."""
    H, psi, ops, ref = cfg3
    x = psi.flat_view()
    errs = {}
    for form in ("fp64", "3xtf32", "bf16x3"):
        y = torch.empty_like(x)
        H.apply_flat(x, y, form)
        errs[form] = _rel(y.cpu().numpy(), ref)
    assert errs["fp64"] <= 1e-12, errs
    assert errs["3xtf32"] <= 2e-5, errs
    assert errs["bf16x3"] <= 2e-5, errs


@pytest.mark.parametrize("form", ["bf16x3", "3xtf32"])
def test_config3_refined_ground_state_against_oracle(cfg3, form):
    """Restarted Lanczos with split-precision Krylov steps and one FP64 refinement per
    restart: the oracle's FP64 matvec applied to the returned vector v gives a Rayleigh
    quotient within 1e-12 of the reported energy and an eigen-residual |Hv - Ev| below
    1e-9 |E| |v|, so an exact eigenvalue of the oracle's operator lies within 1e-9 |E|."""
    H, psi, ops, _ = cfg3
    r = H.lanczos_refined(psi, precision=form, krylov_dim=32, max_restarts=300, tol=1e-12)
    v = r["vec"].flat_view().cpu().numpy()
    hv = OW.heff_matvec(ops, v)
    E_o = float(np.dot(v, hv) / np.dot(v, v))
    res_o = float(np.linalg.norm(hv - E_o * v) / (abs(E_o) * np.linalg.norm(v)))
    assert abs(r["energy"] - E_o) <= 1e-12 * abs(E_o)
    assert res_o <= 1e-9, res_o


def test_config5_gradient_equals_oracle_two_heff_a():
    """d<A|H|A>/dA_k (the hand-written adjoint through torch.autograd) equals 2 H_eff,k A_k
    with the environments and H_eff contracted by the oracle."""
    from cytnx_b200.autodiff import U1MPS

    mps = U1MPS(10, 24, seed=3)
    num = mps.energy(checkpoint_every=4, numerator_only=True)
    g = torch.autograd.grad(num, mps.params)
    bq = [b._qnums[:, 0].copy() for b in mps.bonds]
    bd = [b._degs.copy() for b in mps.bonds]
    flats = [p.detach().cpu().numpy() for p in mps.params]
    for k in range(mps.L):
        ref = 2.0 * OW.mps_heff_times_site(bq, bd, flats, k)
        assert _rel(g[k].cpu().numpy(), ref) <= 1e-12, k
