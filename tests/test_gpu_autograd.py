"""Hand-written adjoint of the block-sparse contraction (torch.autograd.Function) and
the differentiable U(1) MPS energy: gradients against central finite differences and
against 2 H_eff A built with Contract; checkpointed and plain sweeps agree; L-BFGS
lowers the energy."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_contract_adjoint_matches_finite_differences():
    """<G, Contract(A, B)> differentiated by hand vs central differences (h = 1e-6)."""
    from cytnx_b200 import workloads as W
    from cytnx_b200.autodiff import Struct, contract

    spec = W.xxz_spec(24)
    psi, L, M1, M2, R = W.build_two_site(spec, W.xxz_mpo_values(1.0, 1.0), seed=4, device=0)
    a = L._data.clone().requires_grad_(True)
    b = psi._data.clone().requires_grad_(True)
    sa, sb = Struct.of(L.relabel(["w", "a", "ap"])), Struct.of(psi.relabel(["a", "s1", "s2", "b"]))
    out, so = contract(a, sa, b, sb)
    g = torch.randn(out.numel(), dtype=torch.float64, device=out.device, generator=torch.Generator("cuda").manual_seed(1))
    f = torch.dot(out, g)
    ga, gb = torch.autograd.grad(f, (a, b))
    rng = np.random.default_rng(0)
    h = 1e-6
    for x, gx, which in ((a, ga, 0), (b, gb, 1)):
        for i in rng.choice(x.numel(), 16, replace=False):
            xp, xm = x.detach().clone(), x.detach().clone()
            xp[i] += h
            xm[i] -= h
            with torch.no_grad():
                if which == 0:
                    fp = torch.dot(contract(xp, sa, b.detach(), sb)[0], g)
                    fm = torch.dot(contract(xm, sa, b.detach(), sb)[0], g)
                else:
                    fp = torch.dot(contract(a.detach(), sa, xp, sb)[0], g)
                    fm = torch.dot(contract(a.detach(), sa, xm, sb)[0], g)
            fd = float((fp - fm) / (2 * h))
            assert abs(fd - float(gx[i])) < 1e-6 * max(1.0, abs(fd)), (which, i, fd, float(gx[i]))


@pytest.mark.parametrize("L,D", [(10, 16), (32, 512)])
def test_mps_energy_gradient_fd_and_heff(L, D):
    from cytnx_b200.autodiff import U1MPS

    mps = U1MPS(L, D, seed=3)
    E = mps.energy(checkpoint_every=4)
    grads = torch.autograd.grad(E, mps.params)
    flat_g = torch.cat([g.reshape(-1) for g in grads])
    # central finite differences (h = 1e-6, float64) on 64 random entries
    sizes = [p.numel() for p in mps.params]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    rng = np.random.default_rng(7)
    idx = rng.choice(int(offs[-1]), 64, replace=False)
    h = 1e-6
    gmax = float(flat_g.abs().max())
    worst = 0.0
    for gi in idx:
        k = int(np.searchsorted(offs, gi, side="right") - 1)
        i = int(gi - offs[k])
        with torch.no_grad():
            ps = [p.detach() for p in mps.params]
            xp, xm = ps[k].clone(), ps[k].clone()
            xp[i] += h
            xm[i] -= h
            fp = mps.energy([*ps[:k], xp, *ps[k + 1:]], checkpoint_every=0)
            fm = mps.energy([*ps[:k], xm, *ps[k + 1:]], checkpoint_every=0)
        fd = float((fp - fm) / (2 * h))
        worst = max(worst, abs(fd - float(flat_g[gi])))
    assert worst < 1e-6 * max(gmax, 1e-3), (worst, gmax)
    # gradient of <A|H|A> at site k equals 2 H_eff A_k (H_eff from Contract environments)
    num = mps.energy(checkpoint_every=4, numerator_only=True)
    gnum = torch.autograd.grad(num, mps.params)
    for k in (0, L // 2, L - 1):
        y = mps.heff_times_site(k)
        ref = 2.0 * y
        assert float(torch.linalg.vector_norm(gnum[k] - ref) / torch.linalg.vector_norm(ref)) < 1e-11


def test_checkpointed_sweep_equals_plain_sweep():
    from cytnx_b200.autodiff import U1MPS

    mps = U1MPS(12, 24, seed=5)
    E1 = mps.energy(checkpoint_every=4)
    g1 = torch.autograd.grad(E1, mps.params)
    E0 = mps.energy(checkpoint_every=0)
    g0 = torch.autograd.grad(E0, mps.params)
    assert float(E1.detach()) == float(E0.detach())
    for a, b in zip(g1, g0):
        assert torch.allclose(a, b, rtol=1e-12, atol=1e-14)


def test_lbfgs_lowers_the_energy():
    from cytnx_b200.autodiff import U1MPS

    mps = U1MPS(8, 16, seed=1)
    x = torch.cat([p.detach().reshape(-1) for p in mps.params]).clone().requires_grad_(True)
    sizes = [p.numel() for p in mps.params]

    def split(v):
        return list(torch.split(v, sizes))

    opt = torch.optim.LBFGS([x], lr=1.0, max_iter=40, history_size=20, line_search_fn="strong_wolfe",
                            tolerance_grad=1e-12, tolerance_change=1e-15)

    def closure():
        opt.zero_grad()
        e = mps.energy(split(x), checkpoint_every=4)
        e.backward()
        return e

    e0 = float(mps.energy(split(x.detach())))
    opt.step(closure)
    e1 = float(mps.energy(split(x.detach())))
    # exact ground-state energy of the 8-site open Heisenberg chain: -3.374932598687...
    assert e1 < e0 and e1 < -3.3
