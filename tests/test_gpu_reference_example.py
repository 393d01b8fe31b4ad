"""The reference's own two-site U(1) DMRG example, run unmodified with ``cytnx`` bound to
this package (the drop-in check of the Python API).

Mirrors pytests/example/DMRG/dmrg_two_sites_U1_test.py: the script's
``dmrg_XXmodel_U1(Nsites=20, chi=32, numsweeps=6, maxit=2)`` must end within 1e-5 of the
free-fermion energy of the XX chain.  The script is read from a checkout of the reference
given by the environment variable CYTNX_REFERENCE_ROOT (example/DMRG/dmrg_two_sites_U1.py
under it); without one the test is skipped.
"""
import importlib.util
import os
import sys

import numpy as np
import pytest

REF = os.environ.get("CYTNX_REFERENCE_ROOT", "")
SCRIPT = os.path.join(REF, "example", "DMRG", "dmrg_two_sites_U1.py") if REF else ""

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not SCRIPT or not os.path.isfile(SCRIPT),
                                 reason="reference checkout not given (CYTNX_REFERENCE_ROOT)")]


def test_reference_dmrg_two_sites_U1_script_unmodified():
    import cytnx_b200

    saved = sys.modules.get("cytnx")
    sys.modules["cytnx"] = cytnx_b200
    try:
        spec = importlib.util.spec_from_file_location("dmrg_two_sites_U1_reference", SCRIPT)
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        Nsites, chi, numsweeps, maxit = 20, 32, 6, 2
        Es = mod.dmrg_XXmodel_U1(Nsites, chi, numsweeps, maxit)
    finally:
        if saved is None:
            sys.modules.pop("cytnx", None)
        else:
            sys.modules["cytnx"] = saved
    H = np.diag(np.ones(Nsites - 1), k=1) + np.diag(np.ones(Nsites - 1), k=-1)
    D = np.linalg.eigvalsh(H)
    EnExact = 2 * sum(D[D < 0])
    assert np.abs(Es[-1] - EnExact) < 1e-5, (Es[-1], EnExact)
