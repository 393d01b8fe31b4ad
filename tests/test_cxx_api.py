"""The C++ drop-in API (include/cytnx.hpp, namespace cytnx) compiled with g++ and driven by
tests/cxx/two_site_lanczos.cpp: the two-site H_eff through Network / LinOp and
linalg::Lanczos("Gnd"), Tensor permute/contiguous and linalg::Tensordot, against the oracle."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from oracle import workloads as OW

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cxx", "two_site_lanczos.cpp")
LIBDIR = os.path.join(ROOT, "cytnx_b200")


def _compile(out_dir):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libcytnx_b200.so")):
        from cytnx_b200 import build

        build.build()
    exe = os.path.join(str(out_dir), "two_site_lanczos")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-lcytnx_b200", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cxx_api_compiles_and_links(tmp_path):
    """The header is self-contained C++17 and every class/function it uses links."""
    _compile(tmp_path)


@pytest.mark.gpu
def test_cxx_two_site_lanczos_matches_oracle(tmp_path):
    exe = _compile(tmp_path)
    D, iters = 64, 30
    ops = OW.xxz_two_site(D, seed=5)
    q, d = OW.u1_sector_sizes(D)
    mpo = OW.xxz_mpo_values()
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        np.array([len(q)], np.int64).tofile(f)
        np.asarray(q, np.int64).tofile(f)
        np.asarray(d, np.int64).tofile(f)
        np.array([len(mpo)], np.int64).tofile(f)
        for k, v in mpo.items():
            np.asarray(k, np.int64).tofile(f)
            np.array([v], np.float64).tofile(f)
        for name in ("L", "R", "psi"):
            x = ops[name].flat()
            np.array([x.size], np.int64).tofile(f)
            x.astype(np.float64).tofile(f)
        np.array([iters], np.int64).tofile(f)
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(outp)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    raw = open(outp, "rb").read()
    pos = 0

    def vec():
        nonlocal pos
        n = int(np.frombuffer(raw, np.int64, 1, pos)[0])
        pos += 8
        v = np.frombuffer(raw, np.float64, n, pos).copy()
        pos += 8 * n
        return v

    hpsi = vec()
    E = float(np.frombuffer(raw, np.float64, 1, pos)[0])
    pos += 8
    v = vec()
    perm, perm2, td = vec(), vec(), vec()
    threw = int(np.frombuffer(raw, np.int64, 1, pos)[0])

    ref = OW.heff_matvec(ops)
    assert np.linalg.norm(hpsi - ref) <= 1e-12 * np.linalg.norm(ref)
    E_ref, v_ref, it_ref = O.lanczos_gnd_ut(lambda x: OW.heff_matvec(ops, x), ops["psi"].flat(), 1e-300, iters)
    assert it_ref == iters
    assert abs(E - E_ref) <= 1e-10 * abs(E_ref)
    assert min(np.linalg.norm(v - v_ref), np.linalg.norm(v + v_ref)) <= 1e-6 * np.linalg.norm(v_ref)
    a = np.arange(120.0).reshape(4, 3, 5, 2)
    assert np.array_equal(perm, O.permute(a, [3, 1, 0, 2]).ravel())
    assert np.array_equal(perm2, O.permute(O.permute(a, [2, 0, 3, 1]), [1, 0, 3, 2]).ravel())
    b = (0.5 * np.arange(60.0) - 7.0).reshape(5, 2, 6)
    assert np.allclose(td, O.tensordot(a, b, [2, 3], [0, 1]).ravel(), rtol=1e-14, atol=1e-12)
    assert threw == 1
