"""Two-site U(1) DMRG through the cytnx API (tests/dmrg_driver.py) on the GPU.

Mirrors the reference's end-to-end check (pytests/example/DMRG/dmrg_two_sites_U1_test.py:
XX chain, N = 20, chi = 32, 6 sweeps; final energy vs the free-fermion value to 1e-5)."""
import pytest

pytestmark = pytest.mark.gpu


def test_dmrg_xx_chain_network_linop():
    import cytnx_b200 as c
    import dmrg_driver as D

    Es = D.run(c, nsites=20, chi=32, sweeps=6, lanczos_maxiter=4, cvgcrit=1e-12)
    assert abs(Es[-1] - D.free_fermion_energy(20)) < 1e-5, (Es[-1], D.free_fermion_energy(20))


def test_dmrg_planned_heff_matches_network():
    import cytnx_b200 as c
    import dmrg_driver as D

    a = D.run(c, nsites=12, chi=16, sweeps=2, lanczos_maxiter=4, cvgcrit=1e-12)
    b = D.run(c, nsites=12, chi=16, sweeps=2, lanczos_maxiter=4, cvgcrit=1e-12, planned=True)
    assert len(a) == len(b)
    for x, y in zip(a, b):
        assert abs(x - y) < 1e-9 * max(1.0, abs(x))
    assert abs(a[-1] - D.free_fermion_energy(12)) < 1e-4  # 2 sweeps at chi = 16: not fully converged
