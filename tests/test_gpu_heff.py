"""Two-site H_eff matvec and Lanczos: the planned CUDA path against the oracle."""
import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu

NET = {"psi": ["-1", "-2", "-3", "-4"], "L": ["-5", "-1", "0"], "R": ["-7", "-4", "3"],
       "M1": ["-5", "-6", "-2", "1"], "M2": ["-6", "-7", "-3", "2"]}


def to_oracle(u, labels):
    bonds = [O.Bond(b.type(), b._qnums, b._degs) for b in u.bonds()]
    u = u.contiguous()
    blocks = [u.get_block_(i).numpy() for i in range(u.Nblocks())]
    return O.BlockTensor(bonds, labels, u.rowrank(), u._layout.itoi, blocks)


def oracle_heff(ops, order=("L", "M1", "M2", "R")):
    """Pairwise oracle contractions in the given order starting from psi; result in TOUT order."""
    t = ops["psi"]
    for name in order:
        t = ops[name].contract(t) if name == "L" else t.contract(ops[name])
    perm = [t.labels.index(l) for l in ["0", "1", "2", "3"]]
    return t.permute(perm)


def build(D, seed=0):
    from cytnx_b200 import workloads as W

    spec = W.xxz_spec(D)
    return W.build_two_site(spec, W.xxz_mpo_values(1.0, 1.0), seed=seed, device=0)


@pytest.mark.parametrize("D", [16, 64, 256])
def test_heff_matvec_matches_oracle(D):
    import cytnx_b200 as c

    psi, L, M1, M2, R = build(D)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    out = H.matvec(psi)
    ops = {"psi": to_oracle(psi, NET["psi"]), "L": to_oracle(L, NET["L"]), "R": to_oracle(R, NET["R"]),
           "M1": to_oracle(M1, NET["M1"]), "M2": to_oracle(M2, NET["M2"])}
    ref = oracle_heff(ops)
    ref_flat = np.concatenate([b.ravel() for b in ref.blocks])
    assert np.array_equal(ref.itoi, out._layout.itoi)
    got = out.flat_view().cpu().numpy()
    err = np.linalg.norm(got - ref_flat) / np.linalg.norm(ref_flat)
    assert err < 1e-13, err


def test_network_launch_matches_planned_heff():
    """The drop-in path (Network.Launch, default left-fold order) equals the fused plan."""
    import cytnx_b200 as c
    from cytnx_b200 import workloads as W

    psi, L, M1, M2, R = build(64, seed=3)
    net = c.Network()
    net.FromString(W.heff_network_lines())
    net.PutUniTensors(["L", "M1", "M2", "R"], [L, M1, M2, R])
    net.PutUniTensor("psi", psi)
    out_net = net.Launch().contiguous()
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    out = H.matvec(psi)
    a, b = out_net.flat_view(), out.flat_view()
    assert torch.linalg.vector_norm(a - b).item() / torch.linalg.vector_norm(b).item() < 1e-13
    net.setOrder(True, "")
    net._order = None
    out_opt = net.Launch().contiguous()
    assert torch.linalg.vector_norm(out_opt.flat_view() - b).item() / torch.linalg.vector_norm(b).item() < 1e-13


@pytest.mark.parametrize("D", [1024])
def test_heff_hermitian_and_linear(D):
    """Size-independent properties at the benchmark size: <x|Hy> = <Hx|y>, H(ax+y) = aHx + Hy."""
    import cytnx_b200 as c

    psi, L, M1, M2, R = build(D, seed=1)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(H.n, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(H.n, dtype=torch.float64, device="cuda", generator=g)
    hx, hy, hz = torch.empty_like(x), torch.empty_like(x), torch.empty_like(x)
    H.apply_flat(x, hx)
    H.apply_flat(y, hy)
    H.apply_flat(0.3 * x + y, hz)
    lhs, rhs = torch.dot(x, hy).item(), torch.dot(hx, y).item()
    assert abs(lhs - rhs) <= 1e-11 * (abs(lhs) + torch.linalg.vector_norm(hx).item() * torch.linalg.vector_norm(y).item())
    lin = torch.linalg.vector_norm(hz - (0.3 * hx + hy)).item() / torch.linalg.vector_norm(hz).item()
    assert lin < 1e-13


def test_lanczos_heff_matches_oracle():
    import cytnx_b200 as c

    psi, L, M1, M2, R = build(32, seed=2)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    E, vec, it = H.lanczos(psi, maxiter=30, cvgcrit=1e-300)
    ops = {"psi": to_oracle(psi, NET["psi"]), "L": to_oracle(L, NET["L"]), "R": to_oracle(R, NET["R"]),
           "M1": to_oracle(M1, NET["M1"]), "M2": to_oracle(M2, NET["M2"])}
    lay_blocks = [b.shape for b in ops["psi"].blocks]

    def mv(x):
        pos, blocks = 0, []
        for s in lay_blocks:
            n = int(np.prod(s))
            blocks.append(x[pos:pos + n].reshape(s))
            pos += n
        p = O.BlockTensor(ops["psi"].bonds, NET["psi"], 1, ops["psi"].itoi, blocks)
        return np.concatenate([b.ravel() for b in oracle_heff(dict(ops, psi=p)).blocks])

    x0 = psi.flat_view().cpu().numpy()
    E_ref, v_ref, it_ref = O.lanczos_gnd_ut(mv, x0, 1e-300, 30)
    assert it == it_ref == 30
    assert abs(E - E_ref) < 1e-10 * abs(E_ref)
    v = vec.flat_view().cpu().numpy()
    assert min(np.linalg.norm(v - v_ref), np.linalg.norm(v + v_ref)) < 1e-6 * np.linalg.norm(v_ref)
    # the LinOp / callback route gives the same numbers
    E2, vec2 = c.linalg.Lanczos(Hop=H, Tin=psi, method="Gnd", Maxiter=30, CvgCrit=1e-300)
    assert abs(E2.item() - E) < 1e-12 * abs(E)


@pytest.mark.parametrize("precision", ["fp64", "bf16x3"])
def test_lanczos_speculative_matches_callback(precision):
    """ctn_heff2_lanczos_gnd queues each next iteration before the host's tridiagonal solve;
    ctn_lanczos_gnd with a callback around ctn_heff2_matvec runs the same recurrence one
    iteration at a time.  FP64: same energy, iteration count and Ritz vector bit for bit, on a
    run stopped by |dE| < cvgcrit and on one stopped by maxiter.  BF16x3: the planned driver
    takes the matvec result in FP32, so the two routes agree to the FP32 rounding of w (far
    below the split matvec's own error).  The callback route calls the matvec exactly iters
    times."""
    import ctypes

    import cytnx_b200 as c
    from cytnx_b200 import _lib

    psi, L, M1, M2, R = build(32, seed=4)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    H.bind(precision)
    prec = _lib.PRECISIONS[precision]
    x0 = psi.contiguous().flat_view()
    n = H.n
    calls = [0]

    def cb(user, x, y, stream):
        calls[0] += 1
        return _lib.lib().ctn_heff2_matvec(H._h, x, y, prec, stream)

    f = _lib.MATVEC_FN(cb)
    for cvg, maxiter in [(1e-9, 80), (1e-300, 12)]:
        E, vec, it = H.lanczos(psi, maxiter=maxiter, cvgcrit=cvg, precision=precision)
        v = vec.flat_view().clone()
        K = torch.empty((maxiter + 1) * n, dtype=torch.float64, device="cuda")
        work = torch.empty(n + 8 + 1032 + maxiter + 64, dtype=torch.float64, device="cuda")
        eig = torch.empty(n, dtype=torch.float64, device="cuda")
        e2, it2 = ctypes.c_double(), ctypes.c_int()
        calls[0] = 0
        _lib.check(_lib.lib().ctn_lanczos_gnd(f, None, x0.data_ptr(), n, maxiter, cvg, K.data_ptr(),
                                              work.data_ptr(), eig.data_ptr(), ctypes.byref(e2), ctypes.byref(it2),
                                              _lib.stream_ptr()), "ctn_lanczos_gnd")
        torch.cuda.synchronize()
        assert calls[0] == it2.value
        if precision == "fp64":
            assert it2.value == it
            assert (it < maxiter) if cvg > 1e-100 else (it == maxiter)
            assert e2.value == E
            assert torch.equal(eig, v)
        else:
            assert abs(it2.value - it) <= 1 and abs(e2.value - E) <= 1e-7 * abs(E)
            if cvg < 1e-100:
                assert it == it2.value == maxiter
                ov = abs(float(torch.dot(eig, v))) / float(torch.linalg.vector_norm(eig) * torch.linalg.vector_norm(v))
                assert ov > 1 - 1e-6


def test_lanczos_block_golden():
    """tests/linalg_test/Lanczos_Gnd_test.cpp:392-422: E vs Eigh to 1e-12, residual < 1e-6."""
    import cytnx_b200 as c
    from conftest import load_golden

    z = load_golden("lanczos_blocks")
    I = c.Bond(c.BD_IN, [[-1], [0], [1]], [9, 9, 9])
    J = c.Bond(c.BD_OUT, [[-1], [0], [1]], [9, 9, 9])
    Hm = c.UniTensor([I, J], labels=["a", "b"], device=0)
    for i, k in enumerate("ABC"):
        Hm.put_block(c.Tensor.from_numpy(z[k], 0), i)
    Jv = c.Bond(c.BD_OUT, [[-1], [0], [1]], [1, 1, 1])
    guess = c.UniTensor([I, Jv], labels=["b", "c"], device=0)
    rng = np.random.default_rng(1)
    for i in range(3):
        guess.put_block(c.Tensor.from_numpy(rng.standard_normal((9, 1)), 0), i)

    class Op(c.LinOp):
        def matvec(self, v):
            out = c.Contract(Hm, v)
            return out.relabel(["b", "c"])

    E, v = c.linalg.Lanczos(Op("mv", 27), guess, "Gnd", 1e-15, 10000)
    dense = np.zeros((27, 27))
    for i, k in enumerate("ABC"):
        dense[9 * i:9 * i + 9, 9 * i:9 * i + 9] = z[k]
    E0 = np.linalg.eigvalsh(dense).min()
    assert abs(E.item() - E0) < 1e-12
    r = (Op("mv", 27).matvec(v) - E.item() * v).norm()
    assert r < 1e-6


def test_lanczos_dense_arange_golden():
    """tests/linalg_test/Lanczos_Gnd_test.cpp:377-390 (E = -1628.9964650426593, tol 1e-5)."""
    import cytnx_b200 as c

    A = torch.arange(27 * 27, dtype=torch.float64, device="cuda").reshape(27, 27)
    Hd = A + A.T

    class Op(c.LinOp):
        def matvec(self, v):
            return c.Tensor.from_torch(Hd @ v.to_torch())

    E, v = c.linalg.Lanczos(Op("mv", 27), c.arange(27, device=0), "Gnd", 9.999999999999999988e-15, 10000)
    assert abs(E.item() - (-1628.9964650426593)) < 1e-5


@pytest.mark.parametrize("form", ["bf16x3", "3xtf32"])
def test_refined_lanczos_reaches_fp64_energy(form):
    """Split-precision Krylov steps with one FP64 refinement matvec per restart converge to
    the FP64 ground-state energy (same driver run in FP64) far below the matvec error."""
    import cytnx_b200 as c

    psi, L, M1, M2, R = build(128, seed=2)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    ref = H.lanczos_refined(psi, precision="fp64", krylov_dim=24, max_restarts=400, tol=1e-11)
    got = H.lanczos_refined(psi, precision=form, krylov_dim=24, max_restarts=400, tol=1e-11)
    E64, E = ref["energy"], got["energy"]
    assert ref["residual"] <= 1e-11 * abs(E64)
    assert got["residual"] <= 1e-11 * abs(E)  # FP64 eigen-residual of the split-form vector
    assert abs(E - E64) / abs(E64) < 1e-10
    assert got["matvecs_fp64"] == got["restarts"] + 1
    # the returned energy is the FP64 Rayleigh quotient of the returned vector
    v = got["vec"].flat_view()
    hv = torch.empty_like(v)
    H.apply_flat(v, hv, "fp64")
    assert abs(float(torch.dot(v, hv)) - E) < 1e-12 * abs(E)
    assert abs(float(torch.linalg.vector_norm(hv - E * v)) - got["residual"]) < 1e-9 * abs(E)


@pytest.mark.parametrize("n,krydim", [(60, 10), (5, 8)])
def test_refined_lanczos_c_abi_dense_operator(n, krydim):
    """ctn_lanczos_refined through the C ABI with caller matvecs: an FP64 operator for the
    refinement and the same operator with a relative 1e-6 perturbation for the Krylov
    steps.  (5, 8): the Krylov space runs out after five vectors (near-zero beta)."""
    import ctypes

    from cytnx_b200 import _lib

    g = torch.Generator().manual_seed(n)
    A = torch.randn(n, n, generator=g, dtype=torch.float64)
    Hm = ((A + A.T) / 2).cuda()
    noise = torch.randn(n, generator=g, dtype=torch.float64).cuda()
    x0 = torch.randn(n, generator=g, dtype=torch.float64).cuda()
    K = torch.empty(krydim * n, dtype=torch.float64, device="cuda")
    work = torch.empty(n + 3200 + 3 * krydim, dtype=torch.float64, device="cuda")
    eig = torch.empty(n, dtype=torch.float64, device="cuda")
    bufs = (K, work, eig, x0)

    def view(ptr):
        for b in bufs:
            base = b.data_ptr()
            if base <= ptr < base + 8 * b.numel():
                off = (ptr - base) // 8
                return b[off:off + n]
        raise AssertionError("pointer outside the test's buffers")

    def mv_hi(user, x, y, stream):
        view(y).copy_(Hm @ view(x))
        return 0

    def mv_lo(user, x, y, stream):
        xv = view(x)
        view(y).copy_(Hm @ xv + 1e-6 * torch.linalg.vector_norm(xv) * noise)
        return 0

    f_lo, f_hi = _lib.MATVEC_FN(mv_lo), _lib.MATVEC_FN(mv_hi)
    E, res = ctypes.c_double(), ctypes.c_double()
    rs = ctypes.c_int()
    cnt = np.zeros(2, dtype=np.int64)
    _lib.check(_lib.lib().ctn_lanczos_refined(f_lo, None, f_hi, None, x0.data_ptr(), n, krydim, 300, 1e-12,
                                              K.data_ptr(), work.data_ptr(), eig.data_ptr(), ctypes.byref(E),
                                              ctypes.byref(res), ctypes.byref(rs), cnt.ctypes.data_as(_lib.P_i64),
                                              _lib.stream_ptr()), "ctn_lanczos_refined")
    e0 = float(np.linalg.eigvalsh(Hm.cpu().numpy())[0])
    assert abs(E.value - e0) <= 1e-11 * abs(e0)
    assert res.value <= 1e-12 * abs(E.value)
    v = eig.cpu().numpy()
    assert abs(np.linalg.norm(v) - 1.0) < 1e-12
    hv = Hm.cpu().numpy() @ v
    assert np.linalg.norm(hv - E.value * v) <= 2e-12 * abs(E.value)
    assert cnt[1] == rs.value + 1


@pytest.mark.parametrize("form", ["bf16x3", "fp64"])
def test_captured_matvec_graph_replays_eager_bits(form):
    """TwoSiteHeff.capture: a CUDA graph of three matvecs replays the eager result bit for bit
    (also on a new input written into the captured buffer), and re-planning the precision
    (set_tiles) makes the graph refuse to replay."""
    import cytnx_b200 as c
    from cytnx_b200._lib import CytnxError

    psi, L, M1, M2, R = build(256, seed=4)
    H = c.TwoSiteHeff(L, M1, M2, R, psi)
    x = psi.flat_view().clone()
    y = torch.empty_like(x)
    g = H.capture(x, y, form, count=3)
    ref = torch.empty_like(x)
    for seed in (0, 1):
        x.copy_(torch.randn(x.numel(), dtype=torch.float64, device=x.device,
                            generator=torch.Generator(device=x.device).manual_seed(seed)))
        y.zero_()
        g.replay()
        H.apply_flat(x, ref, form)
        torch.cuda.synchronize()
        assert torch.equal(y, ref)
    if form != "fp64":
        H.set_tiles(128, 96, form)
        with pytest.raises(CytnxError, match="stale"):
            g.replay()
