"""Host-side checks of the product library (no GPU needed): the C ABI loads and exports
every declared symbol; block enumeration, the contraction planner, the tridiagonal
eigensolver and the file format agree with the oracle / the reference's goldens."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import oracle as O
from conftest import ROOT, golden_bonds, golden_oracle_tensor, load_golden


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"\b(ctn_\w+)\s*\(", txt):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_all_declared_symbols():
    from cytnx_b200 import _lib

    l = _lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(l, n)]
    assert not missing, missing
    assert l.ctn_version() >= 100
    assert l.ctn_dtype_size(3) == 8 and l.ctn_dtype_size(1) == 16 and l.ctn_dtype_size(99) == 0


def test_bindings_cover_header():
    from cytnx_b200 import _lib

    assert set(_lib.exported_symbols()) <= set(declared_symbols())


@pytest.mark.parametrize("name", ["block_contract_L1", "block_contract_L2", "block_contract_L3",
                                  "block_contract_R3", "block_contract_ans3", "block_permute_T1",
                                  "block_permute_T2", "block_permute_ans2"])
def test_enumeration_matches_golden(name):
    import cytnx_b200 as c

    z = load_golden(name)
    it = c.core.enumerate_blocks(golden_bonds(z, c))
    assert np.array_equal(it, z["itoi"])  # bit-exact index map


def test_enumeration_matches_oracle_u1xz2_and_synthetic():
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    rng = np.random.default_rng(0)
    for trial in range(20):
        r = int(rng.integers(2, 6))
        syms = [c.Symmetry.U1(), c.Symmetry.Zn(2)]
        bonds_c, bonds_o = [], []
        for i in range(r):
            nq = int(rng.integers(1, 5))
            q = np.stack([rng.integers(-3, 4, nq), rng.integers(0, 2, nq)], axis=1)
            d = rng.integers(1, 4, nq)
            t = int(rng.choice([-1, 1]))
            bonds_c.append(c.Bond(t, q, d, syms))
            bonds_o.append(O.Bond(t, q, d, [(-1, 1), (0, 2)]))
        assert np.array_equal(c.core.enumerate_blocks(bonds_c), O.enumerate_blocks(bonds_o))
    spec = W.xxz_spec(1024)
    psi, L, M1, M2, R = W.build_two_site(spec, W.xxz_mpo_values(), seed=0, device=-1)
    for u in (psi, L, R, M1):
        ob = [O.Bond(b.type(), b._qnums, b._degs) for b in u.bonds()]
        assert np.array_equal(u._layout.itoi, O.enumerate_blocks(ob))


def test_tridiag_matches_lapack():
    import cytnx_b200 as c

    rng = np.random.default_rng(5)
    for n in (1, 2, 7, 40):
        d, e = rng.standard_normal(n), rng.standard_normal(n - 1)
        w, z = c.linalg.Tridiag(d, e, True, True)
        wr, zr = O.dstev(d, e) if n > 1 else (d.copy(), np.ones((1, 1)))
        np.testing.assert_allclose(w.numpy(), wr, atol=1e-12)
        zz = z.numpy()
        for j in range(n):
            # eigenvectors are defined up to sign
            s = np.sign(zz[j] @ zr[j])
            np.testing.assert_allclose(s * zz[j], zr[j], atol=1e-9)


def test_contract_planner_flops_match_oracle_pairs():
    """The host planner pairs exactly the block pairs the reference multiplies."""
    import cytnx_b200 as c
    from cytnx_b200.unitensor import contract_plan_flops, structure_only

    for case, labs in [(1, (["a", "b"], ["b", "c"])), (2, (["a", "b"], ["b", "c"])),
                       (3, (["a", "b", "c"], ["c", "d", "e"]))]:
        zl, zr = load_golden(f"block_contract_L{case}"), load_golden(f"block_contract_R{case}")
        A = structure_only(golden_bonds(zl, c), labs[0])
        B = structure_only(golden_bonds(zr, c), labs[1])
        L = golden_oracle_tensor(f"block_contract_L{case}", labs[0])
        R = golden_oracle_tensor(f"block_contract_R{case}", labs[1])
        comm = sorted(set(labs[0]) & set(labs[1]))
        c1 = [labs[0].index(x) for x in comm]
        c2 = [labs[1].index(x) for x in comm]
        expect = 0.0
        for a, ta in enumerate(L.itoi):
            for b, tb in enumerate(R.itoi):
                if all(ta[i] == tb[j] for i, j in zip(c1, c2)):
                    sa, sb = L.blocks[a].shape, R.blocks[b].shape
                    k = np.prod([sa[i] for i in c1])
                    expect += 2.0 * np.prod(sa) / k * np.prod(sb)
        assert contract_plan_flops(A, B) == pytest.approx(expect)


def test_network_parse_and_order():
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    net = c.Network()
    net.FromString(W.heff_network_lines())
    assert net._names == ["psi", "L", "R", "M1", "M2"]
    assert net._tout == ["0", "1", "2", "3"] and net._tout_rowrank == 2
    assert net.getOrder() == "((((psi,L),R),M1),M2)"
    net.setOrder(False, "(((L,psi),M1),(M2,R))")
    assert net._parse_order(net.getOrder()) == ((("L", "psi"), "M1"), ("M2", "R"))


def test_fileio_roundtrip(tmp_path):
    from cytnx_b200 import fileio

    z = load_golden("block_contract_L3")
    import cytnx_b200 as c

    bonds = golden_bonds(z, c)
    d = {"uten_type": 2, "is_braket_form": False, "is_tag": True, "is_diag": False, "rowrank": 1, "name": "x",
         "labels": ["p", "q", "r"],
         "bonds": [{"type": b.type(), "nsym": b.Nsym(), "qnums": b._qnums, "degs": b._degs, "dim": b.dim(),
                    "syms": [{"stype": s.stype, "n": s.n} for s in b.syms()]} for b in bonds],
         "itoi": z["itoi"], "blocks": [np.asarray(b) for b in __import__("conftest").golden_blocks(z)]}
    p = str(tmp_path / "t.cytnx")
    fileio.write_unitensor(p, d)
    e = fileio.read_unitensor(p)
    assert e["labels"] == ["p", "q", "r"] and np.array_equal(e["itoi"], z["itoi"])
    for a, b in zip(e["blocks"], d["blocks"]):
        assert np.array_equal(a, b)


REF_ROOT = os.environ.get("CYTNX_REFERENCE_ROOT", "")


@pytest.mark.skipif(not os.path.isdir(os.path.join(REF_ROOT, "tests", "test_data_base")) or not REF_ROOT,
                    reason="reference checkout not given (CYTNX_REFERENCE_ROOT)")
def test_fileio_reads_reference_files():
    from cytnx_b200 import fileio

    base = os.path.join(REF_ROOT, "tests", "test_data_base", "common", "BlockUniTensor")
    e = fileio.read_unitensor(os.path.join(base, "contract_ans3.cytnx"))
    z = load_golden("block_contract_ans3")
    assert np.array_equal(e["itoi"], z["itoi"])


def test_lanczos_which_argument_errors():
    """The which form's checks and messages (src/linalg/Lanczos.cpp:459-580) run before
    any device work."""
    import cytnx_b200 as c
    from cytnx_b200._lib import CytnxError

    H = c.LinOp("mv", 10, c.Type.Double, c.Device.cuda)
    for kw, msg in ((dict(which="ML"), "'which' should be"), (dict(which="SM"), "'which' should be"),
                    (dict(which="SA", k=0), "k should be >0"), (dict(which="SA", k=11), "k can only be up"),
                    (dict(which="SA", CvgCrit=-1.0), "cvg_crit"), (dict(which="SA", k=3, ncv=4), "ncv should"),
                    (dict(which="SA", ncv=11), "ncv should"), (dict(which="SA", method="Gnd"), "either method")):
        with pytest.raises(CytnxError, match=msg):
            c.linalg.Lanczos(H, None, **kw)
    with pytest.raises(CytnxError, match="Invalid Lanczos method"):
        c.linalg.Lanczos(H, None, "XY")


def test_sym_eigh_matches_numpy():
    import ctypes

    from cytnx_b200 import _lib

    rng = np.random.default_rng(1)
    for n in (1, 2, 7, 40):
        A = rng.standard_normal((n, n))
        A = A + A.T
        w = np.zeros(n)
        z = np.zeros((n, n))
        _lib.check(_lib.lib().ctn_sym_eigh(n, A.ctypes.data_as(_lib.P_dbl), w.ctypes.data_as(_lib.P_dbl),
                                           z.ctypes.data_as(_lib.P_dbl)))
        assert np.abs(np.sort(w) - np.linalg.eigvalsh(A)).max() < 1e-12 * max(1.0, np.abs(w).max())
        assert np.abs(A @ z - z * w).max() < 1e-12 * max(1.0, np.abs(w).max())
        assert np.abs(z.T @ z - np.eye(n)).max() < 1e-13


def test_lanczos_exp_argument_errors():
    import cytnx_b200 as c
    from cytnx_b200._lib import CytnxError

    H = c.LinOp("mv", 10, c.Type.Double, c.Device.cuda)
    with pytest.raises(CytnxError, match="converge criteria must >0"):
        c.linalg.Lanczos_Exp(H, None, -0.1, CvgCrit=0.0)
    with pytest.raises(CytnxError, match="Maxiter must >1"):
        c.linalg.Lanczos_Exp(H, None, -0.1, Maxiter=1)
