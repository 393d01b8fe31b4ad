"""Benchmark: U(1) two-site DMRG H_eff matvec and Lanczos step on B200.

Workload (one GPU): spin-1/2 XXZ (Jz = Jxy = 1) two-site effective Hamiltonian with
U(1) bond dimension D = 4096 (33 sectors q = -16..16, sizes ~ exp(-q^2/72)), MPO bond
dimension 5, seeded ~N(0,1) Hermitian environments -- the precision configuration of
the reference's DMRG path.  A "step" is one H_eff matvec over the resident operands.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--D 4096]

Reported (one JSON line from rank 0):
  value        algorithmic TFLOP/s of the matvec (block-pair GEMM flops of the order
               L -> M1 -> M2 -> R, counted from the block structure) with inputs in HBM
  e2e          the same metric through the public API with psi copied from pinned host
               memory and H psi copied back inside every timed step
  lanczos_s_per_step   seconds per Krylov step of the restarted ground-state Lanczos run
               to convergence (Krylov steps in the headline form, one FP64 refinement
               matvec per restart, FP64 recurrence / re-orthogonalisation / tridiagonal solve)
  dE_rel_vs_fp64       its energy against the same driver run entirely in FP64
  residual_norm_over_x |H x - E x| / |x| of the returned vector, measured in FP64
  roofline     the grouped-GEMM kernel against the measured cuBLAS DGEMM peak
  cpu_baseline the reference algorithm restated on the host cores (oracle), bounded sample
With --gpus N (torchrun) every rank runs an independent replica (the path does not
shard at this size): value = all ranks' flops / max time over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--D", type=int, default=4096)
    ap.add_argument("--lanczos-iters", type=int, default=40)
    ap.add_argument("--cpu-sample-s", type=float, default=15.0)
    ap.add_argument("--precision", default="bf16x3", help="headline arithmetic form: bf16x3, 3xtf32 or fp64")
    ap.add_argument("--matvec-only", action="store_true",
                    help="profiling driver: bind the headline form with --tiles, run warmup + steps matvecs, exit")
    ap.add_argument("--tiles", default="", help="step-1,step-4 tile widths for --matvec-only (e.g. 192,128)")
    ap.add_argument("--epi", default="", help="step-1,step-4 GEMM epilogue forms for --matvec-only / --lanczos-only "
                                             "(0 direct, 1 staged, 2 TMEM fragments; default automatic)")
    ap.add_argument("--lanczos-only", type=int, default=0,
                    help="profiling driver: N restart cycles of the refined Lanczos (headline form, --tiles, "
                         "Krylov dimension 32), the cycles inside a profiler start/stop range, then exit")
    ap.add_argument("--permute-only", action="store_true",
                    help="profiling driver: the large permutes of the permute section, once each, then exit")
    ap.add_argument("--batch-only", type=int, default=0,
                    help="profiling driver: the first N batched Hubbard problems, headline form, --tiles, eager matvecs")
    ap.add_argument("--mps-lbfgs-steps", type=int, default=200,
                    help="differentiable U(1) MPS section (L=32, D=512): L-BFGS steps (0 skips it)")
    ap.add_argument("--batch-problems", type=int, default=256,
                    help="batched Hubbard section: number of two-site problems (0 skips it)")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """SM clocks, power and clock-event (throttle) reasons sampled during the timed region:
    through NVML every 10 ms when the bindings are importable, else nvidia-smi every 200 ms.
    Read-only: no GPU setting is changed."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    _BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.index = index
        self.uuid = None
        try:
            import torch

            u = str(torch.cuda.get_device_properties(index).uuid)
            self.uuid = u if u.startswith("GPU-") else f"GPU-{u}"
            self.index = self.uuid
        except Exception:
            pass
        self.rows = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByUUID(self.uuid) if self.uuid else pynvml.nvmlDeviceGetHandleByIndex(index)
            self._nvml = (pynvml, h)
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        nv, h = self._nvml
        sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
        mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
        try:
            rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
        except Exception:
            rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
        act = lambda k: "Active" if rs & self._BITS[k] else "Not Active"  # noqa: E731
        self.rows.append([str(self.index), str(sm), str(mx), f"{pw:.1f}", hex(rs), act("hw_slowdown"),
                          act("hw_thermal_slowdown"), act("sw_thermal_slowdown"), act("sw_power_cap")])

    def _run(self):
        while not self._stop.is_set():
            try:
                if self._nvml is not None:
                    self._sample_nvml()
                    self._stop.wait(0.01)
                    continue
                r = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                    "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if r.returncode == 0 and r.stdout.strip():
                    self.rows.append([x.strip() for x in r.stdout.strip().split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def quiet_host():
    """One BLAS thread for the oracle from here on: the worker threads a multi-threaded CPU
    baseline leaves behind keep spinning for a while after each call and take host cores from
    the thread that launches the next GPU measurement (host-latency-bound sections such as the
    small dense configuration and the per-phase event profiles are sensitive to it)."""
    if "oracle" in sys.modules:
        sys.modules["oracle"].set_threads(1)


def cpu_baseline_matvec(D, seed, sample_s, threads):
    """Reference CPU algorithm (oracle restatement of BlockUniTensor::contract, OpenBLAS
    dgemm) on the host cores: whole matvecs in the order L -> M1 -> M2 -> R until
    sample_s.  Inputs come from the oracle's own builder (no product code)."""
    import oracle as O
    from oracle import workloads as OW

    O.set_threads(threads)
    ops = OW.xxz_two_site(D, seed=seed)
    outs = OW.heff_chain(ops)  # warm; its results are the step buffers
    n, t0 = 0, time.perf_counter()
    while True:
        OW.heff_chain(ops, outs=outs)
        n += 1
        el = time.perf_counter() - t0
        if el >= sample_s or n >= 50:
            break
    return el / n, n, OW.heff_flops(ops)


def config_for(D, nsec, world):
    """The workload description shared by both arms (the arithmetic form is in ``dtype``)."""
    return {"workload": f"u1_xxz_two_site_heff_D{D}", "D": D, "sectors": nsec, "mpo_bond": 5, "d": 2,
            "order": "L->M1->M2->R", "l2": "inputs larger than L2 (operands + intermediates > 126 MB)",
            "parallelism": f"replicas{world}"}


def run_reference(args, world, rank):
    """The reference's CPU algorithm for the H_eff matvec (the oracle's restatement of
    BlockUniTensor::contract with OpenBLAS dgemm per block pair, all host threads), on
    the same workload, metric and JSON keys as this arm.  A step is one whole matvec
    when --warmup + --steps of them fit in about 150 s; otherwise each step multiplies
    every s-th block pair of all four contractions (s fixed so the run fits, steps
    cycling through the s offsets), i.e. a bounded sample of the matvec, and the flops
    are those of the pairs multiplied.  Imports nothing from the product package."""
    import oracle as O
    from oracle import workloads as OW

    if rank != 0:
        return
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    ops = OW.xxz_two_site(args.D, seed=0)
    nsec = len(OW.u1_sector_sizes(args.D)[0])
    t0 = time.perf_counter()
    outs = OW.heff_chain(ops)  # one untimed whole matvec: sizes the sample, buffers for the steps
    t_full = time.perf_counter() - t0
    stride = max(1, int(np.ceil((args.steps + args.warmup) * t_full / 150.0)))
    for i in range(args.warmup):
        OW.heff_chain(ops, stride=stride, offset=i % stride, outs=outs)
    fl = []
    t0 = time.perf_counter()
    for i in range(args.steps):
        OW.heff_chain(ops, stride=stride, offset=(args.warmup + i) % stride, outs=outs, flops=fl)
    el = time.perf_counter() - t0
    val = sum(fl) / el / 1e12
    sample = (f"{args.steps} whole H_eff matvecs at D={args.D}" if stride == 1 else
              f"{args.steps} steps at D={args.D}, each the block pairs p = offset mod {stride} of the four "
              f"contractions ({sum(fl) / args.steps:.3e} flops per step, a whole matvec is "
              f"{OW.heff_flops(ops):.3e})")
    line = {"metric": METRIC, "impl": "reference", "value": val, "unit": "TFLOP/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": el / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded numpy PCG64)", "config": config_for(args.D, nsec, world),
            "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                             "sample": sample + " (oracle restatement of BlockUniTensor::contract, per-pair "
                                                "permute + OpenBLAS dgemm, as the reference's non-MKL path)"},
            "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


METRIC = "U(1) H_eff matvec TFLOP/s & Lanczos s/step, split-prec vs FP64, dE<=1e-9"


def main():
    args = parse()
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            dist.destroy_process_group()
        return

    from cytnx_b200 import workloads as W

    if args.permute_only:  # one launch per large permute (after one untimed warm launch each)
        out = run_permute(args, torch.device(f"cuda:{local}"), torch.cuda.current_stream(), None, reps=1, small=False)
        print(json.dumps({"permute_only": True, "large": [(o["shape"], o["perm"], o["dtype"]) for o in out["large"]]}))
        return

    if args.batch_only > 0:  # small fixed launch sequence of the batched path for ncu
        from cytnx_b200.batch import BatchedTwoSiteHeff

        dims = W.hubbard_batch_dims(256, seed=0)[: args.batch_only]
        probs = W.hubbard_batch(dims)
        data = [W.problem_data(p, 1000 + i) for i, p in enumerate(probs)]
        tiles = tuple(int(t) for t in args.tiles.split(",")) if args.tiles else (128, 48)
        B = BatchedTwoSiteHeff(probs, args.precision, tiles=tiles)
        B.set_env(B.gather([d[0] for d in data], "L"), B.gather([d[1] for d in data], "R"))
        x = B.gather([d[2] for d in data], "psi")
        y = torch.zeros_like(x)
        for _ in range(args.warmup + args.steps):
            B.matvec(x, y)
        torch.cuda.synchronize()
        print(json.dumps({"batch_only": args.batch_only, "precision": args.precision, "tiles": list(tiles),
                          "workspace_gb": B.workspace_bytes() / 1e9, "out_norm": float(y.norm())}), flush=True)
        return

    spec = W.xxz_spec(args.D)
    mpo_vals = W.xxz_mpo_values(1.0, 1.0, 0.0)
    config_base = config_for(args.D, int(len(spec.dv)), world)

    import ctypes

    import cytnx_b200 as c
    from cytnx_b200 import _lib

    dev = torch.device(f"cuda:{local}")
    st = torch.cuda.current_stream()
    psi, L, M1, M2, R = W.build_two_site(spec, mpo_vals, seed=0, device=local)
    H = c.TwoSiteHeff(L, M1, M2, R, psi, precision=args.precision)
    def fixed_tiles():  # --tiles / --epi of the profiling drivers
        if args.precision == "fp64":
            return
        if args.tiles:
            b1, b4 = (int(t) for t in args.tiles.split(","))
            H.set_tiles(b1, b4, args.precision)
        if args.epi:
            e1, e4 = (int(t) for t in args.epi.split(","))
            _lib.check(_lib.lib().ctn_heff2_set_epilogue(H._h, _lib.PRECISIONS[args.precision], e1, e4), "epi")

    if args.matvec_only:  # small fixed launch sequence for ncu: no autotuning, no other sections
        fixed_tiles()
        x = psi.flat_view()
        y = torch.empty_like(x)
        for _ in range(args.warmup + args.steps):
            H.apply_flat(x, y, args.precision)
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"matvec_only": True, "precision": args.precision, "D": args.D, "tiles": args.tiles,
                              "matvecs": args.warmup + args.steps, "out_norm": float(y.norm())}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.lanczos_only > 0:  # restart cycles of the refined driver inside a profiler range (ncu)
        fixed_tiles()
        H.lanczos_refined(psi, precision=args.precision, krylov_dim=32, max_restarts=2, tol=0.0)  # warm
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        r = H.lanczos_refined(psi, precision=args.precision, krylov_dim=32, max_restarts=args.lanczos_only, tol=0.0)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        if rank == 0:
            print(json.dumps({"lanczos_only": True, "precision": args.precision, "D": args.D,
                              "matvecs_lo": r["matvecs_lo"], "matvecs_fp64": r["matvecs_fp64"],
                              "energy": r["energy"]}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    flops = H.algorithmic_flops()
    tiles = {f: H.autotune(f) for f in ("bf16x3", "3xtf32")}
    x = psi.flat_view()
    forms = [args.precision] + [f for f in ("3xtf32", "bf16x3", "fp64") if f != args.precision]

    def timed_matvecs(form, steps, sampler=None):
        """K matvecs replayed from one CUDA graph (TwoSiteHeff.capture: the same kernels as the
        eager calls without their per-launch host work), W warm-up matvecs from another; also
        the same K matvecs issued eagerly one call at a time, for comparison."""
        y = torch.empty_like(x)
        H.bind(form)
        warm = H.capture(x, y, form, count=max(1, args.warmup))
        run = H.capture(x, y, form, count=steps)
        warm.replay()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if sampler is not None:
            sampler.__enter__()
        e0.record(st)
        run.replay()
        e1.record(st)
        torch.cuda.synchronize()
        if sampler is not None:
            sampler.__exit__(None, None, None)
        y_graph = y.clone()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(st)
        for _ in range(steps):
            H.apply_flat(x, y, form)
        e3.record(st)
        torch.cuda.synchronize()
        if not torch.equal(y, y_graph):
            raise RuntimeError(f"{form}: graph-replayed matvec differs from the eager one")
        t = torch.tensor([e0.elapsed_time(e1), e2.elapsed_time(e3)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        del warm, run
        return float(t[0].item()), y, float(t[1].item())

    def phases(form):
        ms = (ctypes.c_double * 4)()
        nl = ctypes.c_int()
        y = torch.empty_like(x)
        _lib.check(_lib.lib().ctn_heff2_profile(H._h, x.data_ptr(), y.data_ptr(), _lib.PRECISIONS[form], 10, ms,
                                               ctypes.byref(nl), _lib.stream_ptr()), "profile")
        return [ms[i] for i in range(4)], int(nl.value)

    results = {}
    sampler = ClockSampler(local)
    for i, form in enumerate(forms):
        ms, y, ms_eager = timed_matvecs(form, args.steps, sampler if i == 0 else None)
        ph, nl = phases(form)
        results[form] = {"ms_total": ms, "ms_per_matvec": ms / args.steps, "ms_per_matvec_eager": ms_eager / args.steps,
                         "tflops": world * flops * args.steps / (ms * 1e-3) / 1e12, "phase_ms": ph,
                         "launches_per_matvec": nl, "y": y}
    head = results[args.precision]
    value = head["tflops"]

    # matvec error of the split form against the FP64 form (same input)
    y64 = results["fp64"]["y"]
    errs = {f: float((torch.linalg.vector_norm(r["y"] - y64) / torch.linalg.vector_norm(y64)).item())
            for f, r in results.items() if f != "fp64"}
    for f, e in errs.items():
        results[f]["matvec_rel_err_vs_fp64"] = e
    mv_err = errs.get(args.precision)

    # ---- end to end through the public API (pinned host psi in, host H psi out), headline form.
    # Every step copies its input host -> device and its result device -> host.  The copies run
    # on their own streams with three device buffers each, so step i's matvec overlaps the input
    # copy of step i+1 and the output copy of step i-1 (PCIe is full duplex); with two buffers the
    # matvec of step i also waited for the output copy of step i-2 (0.64 vs 0.58 ms per step).
    NBUF = 3
    H.bind(args.precision)
    n_el = x.numel()
    h_in = torch.empty(n_el, dtype=torch.float64, pin_memory=True)
    h_in.copy_(x.cpu())
    h_out = [torch.empty(n_el, dtype=torch.float64, pin_memory=True) for _ in range(NBUF)]
    d_in = [torch.empty(n_el, dtype=torch.float64, device=dev) for _ in range(NBUF)]
    d_out = [torch.empty(n_el, dtype=torch.float64, device=dev) for _ in range(NBUF)]
    s_cmp = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(NBUF)]
    ev_cmp = [torch.cuda.Event() for _ in range(NBUF)]
    ev_out = [torch.cuda.Event() for _ in range(NBUF)]
    used = [False] * NBUF

    def e2e_step(i):
        b = i % NBUF
        if used[b]:
            s_in.wait_event(ev_cmp[b])  # the matvec that read d_in[b] is done
        with torch.cuda.stream(s_in):
            d_in[b].copy_(h_in, non_blocking=True)
            ev_in[b].record(s_in)
        s_cmp.wait_event(ev_in[b])
        if used[b]:
            s_cmp.wait_event(ev_out[b])  # the copy out of d_out[b] is done
        H.apply_flat(d_in[b], d_out[b], args.precision)
        ev_cmp[b].record(s_cmp)
        s_out.wait_event(ev_cmp[b])
        with torch.cuda.stream(s_out):
            h_out[b].copy_(d_out[b], non_blocking=True)
            ev_out[b].record(s_out)
        used[b] = True

    for i in range(4):
        e2e_step(i)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(s_cmp)
    s_in.wait_stream(s_cmp)
    for i in range(args.steps):
        e2e_step(i)
    s_cmp.wait_stream(s_out)
    e3.record(s_cmp)
    torch.cuda.synchronize()
    if not torch.equal(h_out[(args.steps - 1) % NBUF], d_out[(args.steps - 1) % NBUF].cpu()):
        raise RuntimeError("e2e: host output differs from the device result")
    t2 = torch.tensor([e2.elapsed_time(e3)], dtype=torch.float64, device=dev)
    if world > 1:
        dist.all_reduce(t2, op=dist.ReduceOp.MAX)
    e2e_val = world * flops * args.steps / (float(t2.item()) * 1e-3) / 1e12

    # the host link alone: the same two copies per step, on the same streams, with no matvec
    torch.cuda.synchronize()
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(s_cmp)
    s_in.wait_stream(s_cmp)
    s_out.wait_stream(s_cmp)
    for i in range(args.steps):
        with torch.cuda.stream(s_in):
            d_in[i % NBUF].copy_(h_in, non_blocking=True)
        with torch.cuda.stream(s_out):
            h_out[i % NBUF].copy_(d_out[i % NBUF], non_blocking=True)
    s_cmp.wait_stream(s_in)
    s_cmp.wait_stream(s_out)
    e5.record(s_cmp)
    torch.cuda.synchronize()
    link_ms = e4.elapsed_time(e5) / args.steps

    # ---- Lanczos (the reference's Gnd recurrence, fixed iteration count): seconds per step
    lanczos = {}
    for form in forms:
        # warm at the same size: the Krylov buffers come from the caching allocator afterwards
        H.lanczos(psi, maxiter=args.lanczos_iters, cvgcrit=1e-300, precision=form)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        E, vec, it = H.lanczos(psi, maxiter=args.lanczos_iters, cvgcrit=1e-300, precision=form)
        torch.cuda.synchronize()
        lanczos[form] = {"energy": E, "iters": it, "s_per_step": (time.perf_counter() - t0) / max(it, 1)}

    # ---- ground state to convergence: restarted Lanczos, Krylov steps in each form, one FP64
    # refinement matvec per restart; energies are FP64 Rayleigh quotients of the returned vectors
    refined, ground = {}, {}
    for form in forms:
        # warm at the same Krylov dimension (its buffers come from the caching allocator afterwards)
        H.lanczos_refined(psi, precision=form, krylov_dim=32, max_restarts=2, tol=0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = H.lanczos_refined(psi, precision=form, krylov_dim=32, max_restarts=300, tol=1e-12)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        nmv = r["matvecs_lo"] + r["matvecs_fp64"]
        refined[form] = {"energy": r["energy"], "residual_abs": r["residual"],
                         "residual_rel": r["residual"] / abs(r["energy"]), "restarts": r["restarts"],
                         "matvecs_split_or_form": r["matvecs_lo"], "matvecs_fp64": r["matvecs_fp64"],
                         "time_to_solution_s": dt, "s_per_step": dt / max(nmv, 1)}
        ground[form] = r["vec"].flat_view().cpu().numpy()
    e64 = refined["fp64"]["energy"]
    for form in forms:
        refined[form]["dE_rel_vs_fp64"] = abs(refined[form]["energy"] - e64) / abs(e64)
        refined[form]["speedup_vs_fp64"] = refined["fp64"]["time_to_solution_s"] / refined[form]["time_to_solution_s"]

    # ---- peaks for the roofline denominators (cuBLAS, best of 5)
    def gemm_peak(dtype, tf32=False):
        old = torch.backends.cuda.matmul.allow_tf32
        torch.backends.cuda.matmul.allow_tf32 = tf32
        a = torch.randn(8192, 8192, dtype=dtype, device=dev)
        b = torch.randn(8192, 8192, dtype=dtype, device=dev)
        torch.matmul(a, b)
        best = 1e9
        for _ in range(5):
            s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(st)
            torch.matmul(a, b)
            s1.record(st)
            torch.cuda.synchronize()
            best = min(best, s0.elapsed_time(s1))
        torch.backends.cuda.matmul.allow_tf32 = old
        del a, b
        return 2 * 8192 ** 3 / (best * 1e-3) / 1e12

    dgemm_tflops = gemm_peak(torch.float64)
    tf32_tflops = gemm_peak(torch.float32, tf32=True)
    pk, src = peaks()
    prec_id = _lib.PRECISIONS[args.precision]
    if args.precision == "fp64":
        g_flops = _lib.lib().ctn_heff2_gemm_flops(H._h, 1) + _lib.lib().ctn_heff2_gemm_flops(H._h, 4)
        g_ms = head["phase_ms"][1] + head["phase_ms"][3]
        roof = {"bound": "fp64", "achieved": g_flops / (g_ms * 1e-3) / 1e12, "peak": dgemm_tflops,
                "kernel": "k_gemm_grouped_f64 (steps 1 and 4)",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run"}
    else:
        g_flops = _lib.lib().ctn_heff2_split_gemm_flops(H._h, prec_id, 1) + \
            _lib.lib().ctn_heff2_split_gemm_flops(H._h, prec_id, 4)
        g_ms = head["phase_ms"][1] + head["phase_ms"][3]
        tc_peak = tf32_tflops if args.precision == "3xtf32" else float(pk.get("bf16_tflops", 1590.0))
        roof = {"bound": "tensor", "achieved": g_flops / (g_ms * 1e-3) / 1e12, "peak": tc_peak / 3.0,
                "kernel": "k_tc_gemm (tcgen05, steps 1 and 4, stacked per sector)",
                "peak_source": ("cuBLAS TF32 GEMM 8192^3 measured in this run" if args.precision == "3xtf32"
                                else f"MEASURED_PEAKS.json bf16_tflops ({src})") + " / 3 split products"}
    # DRAM bytes (read + write) of the two GEMM launches of one BF16x3 matvec with tiles 192 / 144,
    # from one ncu capture of `bench.py --matvec-only --tiles 192,144` (dram__bytes_read.sum +
    # dram__bytes_write.sum of k_tc_gemm<1,192,2> and k_tc_gemm<1,144,3>)
    traffic = 138.03e6 if (args.precision == "bf16x3" and args.D == 4096) else None
    roof.update({"unit": "TFLOP/s", "frac": roof["achieved"] / roof["peak"], "traffic": traffic,
                 "traffic_unit": "bytes per matvec (steps 1 and 4, ncu capture)",
                 "kernel_flops_per_matvec": g_flops, "kernel_ms_per_matvec": g_ms})
    clocks = sampler.summary()
    quiet_host()
    permute = run_permute(args, dev, st, pk.get("hbm_gbs"))
    quiet_host()
    prec_floor = run_precision_floor(dev) if rank == 0 else None
    fp64_d1024 = run_fp64_d1024(args, dev, st, dgemm_tflops, rank)
    quiet_host()
    config1 = run_config1(args, dev, st, dgemm_tflops) if rank == 0 else None
    quiet_host()
    batched = run_batched(args, world, rank, dev, st) if args.batch_problems > 0 else None
    quiet_host()
    mps_ad = run_mps_autograd(args, dev) if args.mps_lbfgs_steps > 0 else None
    if rank == 0:
        ora = None
        if os.environ.get("CTN_BENCH_NO_ORACLE") != "1":
            ora = oracle_checks(args.D, {f: r["y"].cpu().numpy() for f, r in results.items()}, ground,
                                {f: refined[f]["energy"] for f in forms})
        cpu = None
        if world == 1 and os.environ.get("CTN_BENCH_NO_CPU") != "1":
            threads = os.cpu_count() or 1
            sec, n, oflops = cpu_baseline_matvec(args.D, 0, args.cpu_sample_s, threads)
            cpu = {"value": oflops / sec / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
                   "sample": f"{n} H_eff matvecs at D={args.D} on the host (oracle restatement of "
                             f"BlockUniTensor::contract, OpenBLAS dgemm), {sec:.3f} s each"}
        forms_out = {f: {k: v for k, v in r.items() if k != "y"} for f, r in results.items()}
        line = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": head["ms_per_matvec"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": args.precision, "data": "synthetic (seeded numpy PCG64)",
            "matvec_launch": "the K timed matvecs replayed from one CUDA graph (TwoSiteHeff.capture), "
                             "checked equal to the eager calls; ms_per_step_eager: the same K issued one call "
                             "at a time through TwoSiteHeff.apply_flat",
            "ms_per_step_eager": head["ms_per_matvec_eager"],
            "config": config_base,
            "algorithmic_flops_per_matvec": flops,
            "autotuned_tiles": tiles,
            "forms": forms_out,
            "speedup_vs_fp64": results["fp64"]["ms_per_matvec"] / head["ms_per_matvec"],
            "matvec_rel_err_vs_fp64": mv_err,
            "matvec_rel_err_vs_oracle": ora["matvec_rel_err_vs_oracle"][args.precision] if ora else None,
            "dE_rel_vs_oracle": ora["refined"][args.precision]["dE_rel_vs_oracle"] if ora else None,
            "residual_rel_vs_oracle": ora["refined"][args.precision]["residual_rel_oracle"] if ora else None,
            "oracle_checks": ora,
            "lanczos": lanczos,
            "lanczos_refined": refined,
            "lanczos_s_per_step": refined[args.precision]["s_per_step"],
            "dE_rel_vs_fp64": refined[args.precision]["dE_rel_vs_fp64"],
            "residual_norm_over_x": refined[args.precision]["residual_abs"],
            "e2e": {"value": e2e_val, "unit": "TFLOP/s", "h2d_bytes_per_step": int(x.numel() * 8),
                    "d2h_bytes_per_step": int(x.numel() * 8), "ms_per_step": float(t2.item()) / args.steps,
                    "copies_only_ms_per_step": link_ms,
                    "note": "copies overlap the matvecs; copies_only is the same H2D + D2H pair per step "
                            "with no compute (the host link's duplex time)"},
            "gpu_launches": head["launches_per_matvec"] * args.steps,
            "roofline": roof,
            "peaks": {"hbm_gbs": pk.get("hbm_gbs"), "bf16_tflops": pk.get("bf16_tflops"), "source": src,
                      "dgemm_tflops_measured": dgemm_tflops, "tf32_tflops_measured": tf32_tflops},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "permute": permute,
            "precision_floor": prec_floor,
            "dense_single_site_D64": config1,
            "fp64_D1024": fp64_d1024,
            "batched_hubbard": batched,
            "autograd_mps": mps_ad,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def oracle_checks(D, ys, ground, energies):
    """Errors against the oracle's FP64 matvec, computed on the host outside every timed
    region: each form's matvec output against the oracle's matvec of the same input, and
    each form's refined ground state v checked with the oracle's matvec (Rayleigh quotient
    E_o(v) and eigen-residual |H v - E_o v| / (|E_o| |v|); by the symmetric residual bound an
    exact eigenvalue of the oracle's operator lies within that residual of E_o).  The
    energies' dE is taken against E_o of the FP64 run's ground state."""
    import oracle as O
    from oracle import workloads as OW

    t0 = time.perf_counter()
    O.set_threads(os.cpu_count() or 1)
    ops = OW.xxz_two_site(D, seed=0)
    ref = OW.heff_matvec(ops)
    nref = float(np.linalg.norm(ref))
    out = {"matvec_rel_err_vs_oracle": {f: float(np.linalg.norm(y - ref) / nref) for f, y in ys.items()},
           "refined": {}}
    eo = {}
    for f, v in ground.items():
        hv = OW.heff_matvec(ops, v)
        e = float(np.dot(v, hv) / np.dot(v, v))
        eo[f] = e
        out["refined"][f] = {"E_oracle_rayleigh": e,
                             "residual_rel_oracle": float(np.linalg.norm(hv - e * v) / (abs(e) * np.linalg.norm(v))),
                             "E_reported_minus_E_oracle_rel": abs(energies[f] - e) / abs(e)}
    e_ref = eo.get("fp64")
    for f in out["refined"]:
        out["refined"][f]["dE_rel_vs_oracle"] = abs(energies[f] - e_ref) / abs(e_ref) if e_ref else None
    out["host_seconds"] = time.perf_counter() - t0
    return out


def run_precision_floor(dev, M=512, N=512, K=1408, chunks=(1408, 256, 64, 32)):
    """Where the error of one split-precision product comes from, measured on the device.

    C = A B with A, B ~ N(0, 1) FP64 and K = 1408 (the contraction length of the D=4096 step-4
    GEMM).  For each split form: the relative Frobenius error of the tensor-core GEMM against
    FP64 when K is cut into chunks whose partial products are summed in FP64 (chunk = K: one
    FP32 accumulation over the whole K, the product as the matvec runs it; chunk = one K slice
    of the panel layout: the accumulator leaves FP32 after every slice), and the floor of the
    split representation itself (hi*hi + hi*lo + lo*hi of the same rounded values, summed
    exactly in FP64)."""
    import torch

    from cytnx_b200 import _lib

    g = torch.Generator(device=dev).manual_seed(2024)
    A = torch.randn(M, K, dtype=torch.float64, device=dev, generator=g)
    B = torch.randn(K, N, dtype=torch.float64, device=dev, generator=g)
    ref = A @ B
    nref = torch.linalg.matrix_norm(ref)

    def split_gemm(a, b, p):
        m, k = a.shape
        n = b.shape[1]
        ws = torch.empty(_lib.lib().ctn_split_gemm_workspace_bytes(m, n, k, p), dtype=torch.uint8, device=dev)
        c = torch.empty(m, n, dtype=torch.float64, device=dev)
        _lib.check(_lib.lib().ctn_split_gemm_f64(m, n, k, a.data_ptr(), b.data_ptr(), c.data_ptr(), p, ws.data_ptr(),
                                                 _lib.stream_ptr()), "precision_floor")
        return c

    def tf32(x32):  # round to nearest, ties away (cvt.rna.tf32.f32)
        bits = x32.view(torch.int32)
        return ((bits + 0x1000) & -0x2000).view(torch.float32)

    def rnd(x, form):
        return tf32(x.float()) if form == "3xtf32" else x.to(torch.bfloat16)

    out = {"M": M, "N": N, "K": K}
    for form in ("3xtf32", "bf16x3"):
        p = _lib.PRECISIONS[form]
        row = {}
        for ch in chunks:
            C = torch.zeros_like(ref)
            for k0 in range(0, K, ch):
                C += split_gemm(A[:, k0:k0 + ch].contiguous(), B[k0:k0 + ch].contiguous(), p)
            row[str(ch)] = float((torch.linalg.matrix_norm(C - ref) / nref).item())
        ah = rnd(A, form).double()
        al = rnd(A - ah, form).double()
        bh = rnd(B, form).double()
        bl = rnd(B - bh, form).double()
        rep = ah @ bh + ah @ bl + al @ bh
        out[form] = {"rel_err_by_fp64_chunk": row,
                     "representation_floor": float((torch.linalg.matrix_norm(rep - ref) / nref).item())}
    out["note"] = ("the per-chunk errors fall with the chunk length down to one K slice (the tensor pipe "
                   "accumulates in FP32, so the error of one product grows with K); the 3xTF32 error at one "
                   "K slice is the smallest any FP32-accumulated split product reaches")
    return out


def run_batched(args, world, rank, dev, st):
    """Batched variant: independent two-site Hubbard problems (U=4, t=1, d=4, (N, 2Sz)
    charges, D ~ U[128, 2048]) in FP32, split-precision GEMMs, one launch per phase for all
    problems, replayed from a CUDA graph.  With N ranks the problems are sharded by
    longest-processing-time first (no collective on the data path); time = max over ranks."""
    import torch
    import torch.distributed as dist

    import cytnx_b200 as c
    from cytnx_b200 import _lib
    from cytnx_b200 import workloads as W
    from cytnx_b200.batch import BatchedTwoSiteHeff, problem_flops, shard_problems

    t_setup = time.perf_counter()
    dims = W.hubbard_batch_dims(args.batch_problems, seed=0)
    # cost model for sharding: each problem's algorithmic flops (host planner, every rank alike)
    all_probs = W.hubbard_batch(dims)
    mine = shard_problems([problem_flops(p) for p in all_probs], world)[rank]
    probs = [all_probs[i] for i in mine]
    data = [W.problem_data(p, 1000 + i) for p, i in zip(probs, mine)]
    out = {"problems": args.batch_problems, "D_range": [128, 2048], "model": "Hubbard U=4 t=1, d=4, (N,2Sz) U(1)xU(1)",
           "sector_sigma": 4.0, "io_dtype": "f32", "shards": world, "forms": {}}
    steps = max(args.steps, 10)
    for form, cand1, cand4 in (("bf16x3", (96, 128, 192), (32, 48, 64)), ("3xtf32", (96, 128, 192), (32, 48, 64))):
        B = BatchedTwoSiteHeff(probs, form)
        L_all = B.gather([d[0] for d in data], "L")
        R_all = B.gather([d[1] for d in data], "R")
        x_all = B.gather([d[2] for d in data], "psi")
        B.set_env(L_all, R_all)
        tune = B.autotune(x_all, step1=cand1, step4=cand4, reps=3)
        y = torch.zeros_like(x_all)
        B.capture(x_all, y)
        for _ in range(args.warmup):
            B.replay()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(steps):
            B.replay()
        e1.record(st)
        torch.cuda.synchronize()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item()) / steps
        ph = B.profile(x_all, torch.zeros_like(x_all), 5)
        gf = torch.tensor([B.gemm_flops()], dtype=torch.float64, device=dev)
        if world > 1:
            dist.all_reduce(gf)
        gst = B.gemm_stats()
        # algorithmic bytes: every problem's FP32 environments and vector read once, the result
        # written once; the GEMM panels (hi + lo) are the implementation's operand traffic
        alg_bytes = 4.0 * sum(L_._layout.nelem + R_._layout.nelem + 2 * P_._layout.nelem
                              for (L_, _, _, R_, P_) in probs)
        out["forms"][form] = {"ms_per_batch": ms, "matvecs_per_s": args.batch_problems / (ms * 1e-3),
                              "useful_tflops": float(gf.item()) / (ms * 1e-3) / 1e12, "phase_ms": ph,
                              "tiles": [tune["step1"], tune["step4"]], "graph_replay": True,
                              "launches_per_batch": 4, "workspace_gb": B.workspace_bytes() / 1e9,
                              "gemm_stats_rank0": gst,
                              "roofline": {
                                  "algorithmic_bytes_per_batch_rank0": alg_bytes,
                                  "step4_panel_bytes_over_operand_bytes":
                                      gst["step4"]["panel_bytes"] / max(1.0, gst["step4"]["operand_bytes"]),
                                  "step1_panel_bytes_over_operand_bytes":
                                      gst["step1"]["panel_bytes"] / max(1.0, gst["step1"]["operand_bytes"]),
                                  "executed_over_useful_flops": (gst["step1"]["executed_flops"] +
                                                                 gst["step4"]["executed_flops"]) /
                                                                (gst["step1"]["useful_flops"] +
                                                                 gst["step4"]["useful_flops"]),
                                  "step4_ms": ph[3], "step4_panel_GB_s": gst["step4"]["panel_bytes"] / (ph[3] * 1e-3) / 1e9},
                              "_B": B, "_y": y}
    # per-problem error of each form against the FP64 planned matvec of the same (FP32-valued) inputs
    errs = {f: [] for f in out["forms"]}
    for i, ((L, M1, M2, R, psi), (l, r, x)) in enumerate(zip(probs, data)):
        Lg, Rg, Pg = W.materialize(L, l, dev), W.materialize(R, r, dev), W.materialize(psi, x, dev)
        H = c.TwoSiteHeff(Lg, M1, M2, Rg, Pg)
        ref = H.matvec(Pg).flat_view()
        nref = torch.linalg.vector_norm(ref)
        for f, rec in out["forms"].items():
            got = rec["_B"].slice(rec["_y"], i).double()
            errs[f].append(float((torch.linalg.vector_norm(got - ref) / nref).item()))
        del H
    # a sample of the problems against the oracle's FP64 matvec (host, untimed, rank 0's shard)
    from oracle import workloads as OW

    pick = list(range(0, len(probs), max(1, len(probs) // 8)))[:8]
    oerr = {f: [] for f in out["forms"]}
    for i in pick:
        ref = OW.heff_matvec(OW.hubbard_two_site(dims[mine[i]], 1000 + mine[i]))
        nref = np.linalg.norm(ref)
        for f, rec in out["forms"].items():
            got = rec["_B"].slice(rec["_y"], i).double().cpu().numpy()
            oerr[f].append(float(np.linalg.norm(got - ref) / nref))
    for f, rec in out["forms"].items():
        rec["rel_err_vs_oracle_sample"] = {"problems": [int(mine[i]) for i in pick],
                                           "D": [int(dims[mine[i]]) for i in pick], "max": max(oerr[f])}
    for f, rec in out["forms"].items():
        e = torch.tensor(errs[f], dtype=torch.float64, device=dev)
        mx = e.max().clone()
        if world > 1:
            dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        rec["rel_err_vs_fp64_max"] = float(mx.item())
        rec["rel_err_vs_fp64_median_rank0"] = float(e.median().item())
        del rec["_B"], rec["_y"]
    if rank == 0 and os.environ.get("CTN_BENCH_NO_CPU") != "1":
        # CPU baseline: the oracle's FP64 matvec (BlockUniTensor::contract restated, OpenBLAS, all
        # host threads) looping over problems of this batch for ~10 s; the batch time is the
        # sampled time scaled by the batch's algorithmic flops over the sample's
        import oracle as O
        from oracle import workloads as OW

        O.set_threads(os.cpu_count() or 1)
        t_c, f_c, done, t0 = 0.0, 0.0, [], time.perf_counter()
        for i in range(len(mine)):
            ops = OW.hubbard_two_site(dims[mine[i]], 1000 + mine[i])
            ta = time.perf_counter()
            OW.heff_matvec(ops)
            t_c += time.perf_counter() - ta
            f_c += OW.heff_flops(ops)
            done.append(int(mine[i]))
            if time.perf_counter() - t0 > 10.0:
                break
        out["cpu_baseline"] = {"matvecs_per_s": len(done) / t_c, "tflops": f_c / t_c / 1e12,
                               "sampled_problems": done, "sampled_D": [int(dims[i]) for i in done],
                               "batch_mean_D": float(np.mean(dims)), "seconds": t_c, "flops": f_c,
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": "oracle FP64 matvecs (BlockUniTensor::contract restated, OpenBLAS dgemm) "
                                         "over the first problems of the batch for about 10 s"}
    out["setup_s"] = time.perf_counter() - t_setup
    return out


def run_fp64_d1024(args, dev, st, dgemm_tflops, rank):
    """Plain FP64 U(1) configuration: two-site XXZ H_eff at D=1024, 40 Lanczos iterations
    (the reference's Gnd recurrence) and the block SVD truncation of the ground state back
    to D (Svd_truncate, rowrank 2: (a, s1) | (s2, b)).  Roofline: the grouped FP64 DMMA GEMMs
    of steps 1 and 4 against the measured cuBLAS DGEMM.  CPU baseline (rank 0): the oracle's
    matvec (BlockUniTensor::contract restated, OpenBLAS), its Lanczos_Gnd_Ut and its block
    Svd_truncate on all host threads."""
    import ctypes

    import torch

    import cytnx_b200 as c
    from cytnx_b200 import _lib
    from cytnx_b200 import workloads as W

    spec = W.xxz_spec(1024)
    mpo = W.xxz_mpo_values(1.0, 1.0, 0.0)
    psi, L, M1, M2, R = W.build_two_site(spec, mpo, seed=0, device=dev.index)
    H = c.TwoSiteHeff(L, M1, M2, R, psi, precision="fp64")
    flops = H.algorithmic_flops()
    x = psi.flat_view()
    y = torch.empty_like(x)
    for _ in range(5):
        H.apply_flat(x, y, "fp64")
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 200
    e0.record(st)
    for _ in range(reps):
        H.apply_flat(x, y, "fp64")
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # the same matvecs replayed from a CUDA graph (the three kernels of a D=1024 matvec are short
    # enough that host-issued back-to-back calls can be limited by the host's launch rate)
    ms_graph = None
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, capture_error_mode="thread_local"):
            for _ in range(20):
                H.apply_flat(x, y, "fp64")
        g.replay()
        torch.cuda.synchronize()
        e0.record(st)
        for _ in range(reps // 20):
            g.replay()
        e1.record(st)
        torch.cuda.synchronize()
        ms_graph = e0.elapsed_time(e1) / (reps // 20 * 20)
        del g
    except Exception as ex:  # report the host-issued figure alone
        print(f"[bench] fp64_D1024 graph replay unavailable: {ex}", file=sys.stderr)
    ph = (ctypes.c_double * 4)()
    nl = ctypes.c_int()
    _lib.check(_lib.lib().ctn_heff2_profile(H._h, x.data_ptr(), y.data_ptr(), 0, 20, ph, ctypes.byref(nl),
                                           _lib.stream_ptr()), "profile")
    g_flops = _lib.lib().ctn_heff2_gemm_flops(H._h, 1) + _lib.lib().ctn_heff2_gemm_flops(H._h, 4)
    g_ms = ph[1] + ph[3]
    H.lanczos(psi, maxiter=4, cvgcrit=1e-300)  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    E, vec, it = H.lanczos(psi, maxiter=40, cvgcrit=1e-300)
    torch.cuda.synchronize()
    t_lan = time.perf_counter() - t0
    vec.set_rowrank_(2)
    c.linalg.Svd_truncate(vec, 1024)  # warm (cuSOLVER handles)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    S, U, Vt = c.linalg.Svd_truncate(vec, 1024)
    torch.cuda.synchronize()
    t_svd = time.perf_counter() - t0
    s = S.flat_view()
    kept = int(S.shape()[0])
    out = {"workload": "u1_xxz_two_site_heff_D1024_fp64", "algorithmic_flops_per_matvec": flops,
           "matvec_ms": ms, "matvec_tflops": flops / (ms * 1e-3) / 1e12,
           "matvec_ms_graph": ms_graph,
           "matvec_tflops_graph": flops / (ms_graph * 1e-3) / 1e12 if ms_graph else None,
           "phase_ms": [ph[i] for i in range(4)],
           "lanczos_iters": it, "lanczos_s_per_step": t_lan / max(it, 1), "energy_40": E,
           "svd_truncate_s": t_svd, "svd_kept": kept, "svd_norm2_kept": float((s * s).sum().item()),
           "roofline": {"bound": "fp64 tensor (DMMA)", "kernel": "k_gemm_grouped_f64 (steps 1 and 4)",
                        "achieved": g_flops / (g_ms * 1e-3) / 1e12, "peak": dgemm_tflops, "unit": "TFLOP/s",
                        "frac": g_flops / (g_ms * 1e-3) / 1e12 / dgemm_tflops,
                        "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                        "kernel_flops_per_matvec": g_flops, "kernel_ms_per_matvec": g_ms}}
    if rank == 0 and os.environ.get("CTN_BENCH_NO_CPU") != "1":
        import oracle as O
        from oracle import svd as OS
        from oracle import workloads as OW

        O.set_threads(os.cpu_count() or 1)
        ops = OW.xxz_two_site(1024, seed=0)
        outs = OW.heff_chain(ops)
        n, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < 3.0:
            OW.heff_chain(ops, outs=outs)
            n += 1
        cpu_mv = (time.perf_counter() - t0) / n
        t0 = time.perf_counter()
        E_o, v_o, it_o = O.lanczos_gnd_ut(lambda z: OW.heff_matvec(ops, z), ops["psi"].flat(), 1e-300, 40)
        cpu_lan = (time.perf_counter() - t0) / it_o
        vo = OW.with_psi(ops, v_o)["psi"]
        vo = O.BlockTensor(vo.bonds, vo.labels, 2, vo.itoi, vo.blocks)
        t0 = time.perf_counter()
        So, _, _, _ = OS.svd_truncate(vo, 1024)
        cpu_svd = time.perf_counter() - t0
        out["energy_40_oracle"] = E_o
        out["dE_rel_vs_oracle"] = abs(E - E_o) / abs(E_o)
        out["cpu_baseline"] = {"matvec_ms": cpu_mv * 1e3, "matvec_tflops": flops / cpu_mv / 1e12,
                               "lanczos_s_per_step": cpu_lan, "svd_truncate_s": cpu_svd,
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"{n} oracle matvecs (3 s), 40 oracle Lanczos_Gnd_Ut iterations, one "
                                         "oracle block Svd_truncate (numpy LAPACK per sector)"}
    return out


def run_config1(args, dev, st, dgemm_tflops):
    """Plain dense FP64 single-site configuration: L[64,5,64], R[64,5,64] (symmetrised over the
    two bond indices), the XXZ MPO W[5,5,2,2], A[64,2,64]; the matvec through Network / LinOp
    (the drop-in path) and 30 iterations of linalg.Lanczos("Gnd").  CPU baseline: the same
    matvec as three oracle Tensordot calls (Tensordot.cpp:29-110, OpenBLAS dgemm, all host
    threads) inside the oracle's Lanczos_Gnd_Ut restatement."""
    import torch

    import cytnx_b200 as c
    import oracle as O
    from cytnx_b200 import workloads as W

    D = 64
    rng = np.random.default_rng(0)
    L = rng.standard_normal((D, 5, D))
    L = 0.5 * (L + L.transpose(2, 1, 0))
    R = rng.standard_normal((D, 5, D))
    R = 0.5 * (R + R.transpose(2, 1, 0))
    Wm = np.zeros((5, 5, 2, 2))
    for (a, b, s_, sp), v in W.xxz_mpo_values(1.0, 1.0, 0.0).items():
        Wm[a, b, s_, sp] = v
    A = rng.standard_normal((D, 2, D))
    A /= np.linalg.norm(A)
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
    # flops of the three pairwise contractions (L.A over a; .W over (w, s); .R over (b, w2))
    flops = 2.0 * (5 * D) * (2 * D) * D + 2.0 * (D * D) * (5 * 2) * (5 * 2) + 2.0 * (D * 2) * D * (D * 5)
    for _ in range(5):
        H.matvec(Au)
    torch.cuda.synchronize()
    reps = 200
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(st)
    for _ in range(reps):
        H.matvec(Au)
    e1.record(st)
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / reps
    dev_ms = e0.elapsed_time(e1) / reps
    c.linalg.Lanczos(Hop=H, Tin=Au, method="Gnd", Maxiter=30, CvgCrit=1e-300)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    E, _ = c.linalg.Lanczos(Hop=H, Tin=Au, method="Gnd", Maxiter=30, CvgCrit=1e-300)
    torch.cuda.synchronize()
    lan_s = (time.perf_counter() - t0) / 30
    # CPU: the reference's dense path (three Tensordot calls) and its Lanczos
    O.set_threads(os.cpu_count() or 1)

    def mv(x):
        a = x.reshape(D, 2, D)
        t = O.tensordot(L, a, [0], [0])            # [w, ap, s, b]
        t = O.tensordot(t, Wm, [0, 2], [0, 2])      # [ap, b, w2, sp]
        t = O.tensordot(t, R, [1, 2], [0, 1])       # [ap, sp, bp]
        return t.reshape(-1)

    mv(A.reshape(-1))
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < 2.0:
        mv(A.reshape(-1))
        n += 1
    cpu_mv = (time.perf_counter() - t0) / n
    t0 = time.perf_counter()
    E_ref, _, it = O.lanczos_gnd_ut(mv, A.reshape(-1), 1e-300, 30)
    cpu_lan = (time.perf_counter() - t0) / it
    return {"workload": "dense_fp64_single_site_D64", "algorithmic_flops_per_matvec": flops,
            "matvec_ms_wall": wall * 1e3, "matvec_ms_device": dev_ms,
            "matvec_gflops_wall": flops / wall / 1e9,
            "lanczos_iters": 30, "lanczos_s_per_step": lan_s, "energy_30": float(E.item()),
            "energy_30_oracle": float(E_ref), "dE_rel_vs_oracle": abs(float(E.item()) - E_ref) / abs(E_ref),
            "roofline": {"bound": "launch / host latency (1.1e7 flops per matvec through three "
                                  "Network contractions)",
                         "achieved_tflops": flops / (dev_ms * 1e-3) / 1e12, "peak_tflops": dgemm_tflops,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run",
                         "frac": flops / (dev_ms * 1e-3) / 1e12 / dgemm_tflops},
            "cpu_baseline": {"matvec_ms": cpu_mv * 1e3, "matvec_gflops": flops / cpu_mv / 1e9,
                             "lanczos_s_per_step": cpu_lan, "cores": os.cpu_count() or 1, "kind": "port",
                             "sample": "the matvec as three oracle Tensordot calls (permute + OpenBLAS dgemm) "
                                       "for 2 s, then 30 iterations of the oracle Lanczos_Gnd_Ut"}}


def run_permute(args, dev, st, hbm_peak, reps=None, small=True):
    """Tensor permute + contiguous (ctn_permute): the configuration's 24 permutations of a
    [64,2,2,64] float64 tensor (L2-resident, launch-latency bound) and HBM-bound
    transposes of 512 MB tensors; GB/s = 2 x bytes / device time."""
    import itertools

    import torch

    from cytnx_b200 import _lib

    lib = _lib.lib()

    def timed(x, perm, reps):
        y = torch.empty_like(x)
        did = {torch.float64: 3, torch.float32: 4, torch.int16: 9}[x.dtype]
        osh = np.array(x.shape, dtype=np.uint64)
        mp = np.array(perm, dtype=np.uint64)

        def go():
            _lib.check(lib.ctn_permute(x.data_ptr(), y.data_ptr(), did, x.dim(), osh.ctypes.data_as(_lib.P_u64),
                                       mp.ctypes.data_as(_lib.P_u64), _lib.stream_ptr()), "permute")
        go()
        torch.cuda.synchronize()
        if not torch.equal(y.reshape(-1), x.permute(*perm).contiguous().reshape(-1)):
            raise RuntimeError(f"permute mismatch for {tuple(x.shape)} {perm}")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            go()
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        return ms, 2 * x.numel() * x.element_size() / (ms * 1e-3) / 1e9

    out = {"small": {}, "large": []}
    x = torch.randn(64, 2, 2, 64, dtype=torch.float64, device=dev)
    tot = 0.0
    for perm in itertools.permutations(range(4)) if small else ():
        ms, _ = timed(x, perm, reps or 200)
        tot += ms
    if small:
        # device-only time of the 24 launches: the same calls captured once in a CUDA graph
        ys = [torch.empty_like(x) for _ in range(24)]
        osh = np.array(x.shape, dtype=np.uint64)
        mps_ = [np.array(p, dtype=np.uint64) for p in itertools.permutations(range(4))]
        gs = torch.cuda.Stream()
        gs.wait_stream(torch.cuda.current_stream())
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.stream(gs):
            for y, mp in zip(ys, mps_):  # warm outside the capture
                _lib.check(lib.ctn_permute(x.data_ptr(), y.data_ptr(), 3, 4, osh.ctypes.data_as(_lib.P_u64),
                                           mp.ctypes.data_as(_lib.P_u64), _lib.stream_ptr()), "permute")
            with torch.cuda.graph(graph, stream=gs):
                for y, mp in zip(ys, mps_):
                    _lib.check(lib.ctn_permute(x.data_ptr(), y.data_ptr(), 3, 4, osh.ctypes.data_as(_lib.P_u64),
                                               mp.ctypes.data_as(_lib.P_u64), _lib.stream_ptr()), "permute")
        torch.cuda.synchronize()
        for _ in range(3):
            graph.replay()
        torch.cuda.synchronize()
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        nrep = 50
        g0.record(st)
        for _ in range(nrep):
            graph.replay()
        g1.record(st)
        torch.cuda.synchronize()
        dev_us = g0.elapsed_time(g1) / nrep / 24 * 1e3
        for y, mp in zip(ys, mps_):
            if not torch.equal(y.reshape(-1), x.permute(*[int(v) for v in mp]).contiguous().reshape(-1)):
                raise RuntimeError("graph-replayed permute mismatch")
        del graph
        # CPU baseline: the oracle's Movemem_cpu loop on the same 24 permutations
        import oracle as O

        xh = x.cpu().numpy()
        t0 = time.perf_counter()
        nrep_c = 20
        for _ in range(nrep_c):
            for p in itertools.permutations(range(4)):
                O.permute(xh, p)
        cpu_us = (time.perf_counter() - t0) / (nrep_c * 24) * 1e6
    out["small"] = {"shape": [64, 2, 2, 64], "dtype": "f64", "perms": 24, "total_ms_24": tot,
                    "mean_us_per_perm": tot / 24 * 1e3, "bytes_per_perm": 2 * x.numel() * 8}
    if small:
        out["small"].update({"device_us_per_perm_graph": dev_us,
                             "device_GB_s_graph": 2 * x.numel() * 8 / (dev_us * 1e-6) / 1e9,
                             "note": "mean_us_per_perm is host-issued (ctypes call + launch each); the graph "
                                     "figure is the same 24 launches replayed from one CUDA graph",
                             "cpu_baseline_us_per_perm": cpu_us,
                             "cpu_baseline": "oracle restatement of Movemem_cpu.cpp:152-191 (1 thread)"})
    for shape, perm, dt in (((2048, 4, 4, 2048), (3, 1, 2, 0), torch.float64),
                            ((2048, 4, 4, 2048), (0, 2, 1, 3), torch.float64),
                            ((2048, 4, 4, 2048), (1, 0, 3, 2), torch.float64),
                            ((4096, 4, 4, 4096), (3, 1, 2, 0), torch.float32),
                            ((4096, 4, 4, 4096), (3, 1, 2, 0), torch.int16)):
        xl = (torch.randn(*shape, device=dev) * 100).to(dt)
        ms, gbs = timed(xl, perm, reps or 20)
        out["large"].append({"shape": list(shape), "perm": list(perm), "dtype": str(dt).replace("torch.", ""),
                             "ms": ms, "GB_s": gbs, "frac_of_hbm": gbs / hbm_peak if hbm_peak else None})
        del xl
    return out


def run_mps_autograd(args, dev):
    """Differentiation variant: finite U(1) MPS, L=32, D=512, d=2, XXZ MPO; energy
    <A|H|A>/<A|A> through block-sparse contractions with the hand-written adjoint,
    environments checkpointed every 4 sites; gradient checks, then L-BFGS."""
    import torch

    from cytnx_b200.autodiff import U1MPS

    L, D = 32, 512
    t_setup = time.perf_counter()
    mps = U1MPS(L, D, seed=0, device=dev)
    out = {"L": L, "D": D, "d": 2, "model": "XXZ Jz=1 Jxy=1 h=0", "params": mps.numel(), "checkpoint_every": 4}
    for ce in (4, 0):  # warm both forms, then time one energy + gradient each and record peak memory
        E = mps.energy(checkpoint_every=ce)
        torch.autograd.grad(E, mps.params)
        torch.cuda.synchronize()
        torch.cuda.reset_peak_memory_stats(dev)
        t0 = time.perf_counter()
        E = mps.energy(checkpoint_every=ce)
        g = torch.autograd.grad(E, mps.params)
        torch.cuda.synchronize()
        out[f"eval_grad_s_ckpt{ce}"] = time.perf_counter() - t0
        out[f"peak_mem_mb_ckpt{ce}"] = torch.cuda.max_memory_allocated(dev) / 1e6
    flat_g = torch.cat([x.reshape(-1) for x in g])
    sizes = [p.numel() for p in mps.params]
    offs = np.concatenate([[0], np.cumsum(sizes)])
    rng = np.random.default_rng(7)
    h, worst = 1e-6, 0.0
    for gi in rng.choice(int(offs[-1]), 64, replace=False):
        k = int(np.searchsorted(offs, gi, side="right") - 1)
        i = int(gi - offs[k])
        with torch.no_grad():
            ps = [p.detach() for p in mps.params]
            xp, xm = ps[k].clone(), ps[k].clone()
            xp[i] += h
            xm[i] -= h
            fd = float((mps.energy([*ps[:k], xp, *ps[k + 1:]], checkpoint_every=0) -
                        mps.energy([*ps[:k], xm, *ps[k + 1:]], checkpoint_every=0)) / (2 * h))
        worst = max(worst, abs(fd - float(flat_g[gi])))
    out["fd_check"] = {"entries": 64, "h": h, "max_abs_err": worst, "max_abs_grad": float(flat_g.abs().max())}
    num = mps.energy(checkpoint_every=4, numerator_only=True)
    gnum = torch.autograd.grad(num, mps.params)
    # 2 H_eff,k A_k from the oracle's contractions (environments included), host, untimed
    import oracle as O
    from oracle import workloads as OW

    O.set_threads(os.cpu_count() or 1)
    bq = [b._qnums[:, 0].copy() for b in mps.bonds]
    bd = [b._degs.copy() for b in mps.bonds]
    flats = [p.detach().cpu().numpy() for p in mps.params]
    errs = []
    for k in (0, L // 2, L - 1):
        ref = 2.0 * OW.mps_heff_times_site(bq, bd, flats, k)
        errs.append(float(np.linalg.norm(gnum[k].cpu().numpy() - ref) / np.linalg.norm(ref)))
    out["grad_vs_oracle_2HeffA_rel_err_max"] = max(errs)
    out["grad_vs_oracle_2HeffA_sites"] = [0, L // 2, L - 1]
    # CPU baseline: the same energy and gradient by the oracle's environment sweeps (pairwise
    # contractions restating BlockUniTensor::contract, OpenBLAS), all host threads
    t0 = time.perf_counter()
    num_o, den_o, g_o = OW.mps_energy_grad(bq, bd, flats)
    cpu_s = time.perf_counter() - t0
    with torch.no_grad():
        E_gpu = float(mps.energy(checkpoint_every=4))
    gd = torch.autograd.grad(mps.energy(checkpoint_every=4), mps.params)
    gerr = max(float(np.linalg.norm(gd[k].cpu().numpy() - g_o[k]) / max(np.linalg.norm(g_o[k]), 1e-300))
               for k in (0, L // 2, L - 1))
    out["cpu_baseline"] = {"eval_grad_s": cpu_s, "cores": os.cpu_count() or 1, "kind": "port",
                           "sample": "one energy + gradient of the L=32, D=512 MPS by the oracle's left/right "
                                     "environment sweeps (BlockUniTensor::contract restated, OpenBLAS)",
                           "energy_rel_diff_vs_gpu": abs(num_o / den_o - E_gpu) / abs(E_gpu),
                           "grad_rel_diff_vs_gpu_max": gerr}
    if args.mps_lbfgs_steps > 0:
        x = torch.cat([p.detach().reshape(-1) for p in mps.params]).clone().requires_grad_(True)
        opt = torch.optim.LBFGS([x], lr=1.0, max_iter=args.mps_lbfgs_steps, history_size=30,
                                line_search_fn="strong_wolfe", tolerance_grad=1e-14, tolerance_change=1e-16)
        hist = []

        def closure():
            opt.zero_grad()
            e = mps.energy(list(torch.split(x, sizes)), checkpoint_every=4)
            e.backward()
            hist.append(float(e.detach()))
            return e

        t0 = time.perf_counter()
        opt.step(closure)
        torch.cuda.synchronize()
        st = opt.state[opt._params[0]]
        out["lbfgs"] = {"steps": int(st.get("n_iter", 0)), "energy_evals": int(st.get("func_evals", len(hist))),
                        "seconds": time.perf_counter() - t0, "energy_initial": hist[0], "energy_final": hist[-1],
                        "energy_per_site_final": hist[-1] / L,
                        "trace_every_20": hist[::20]}
    out["setup_and_checks_s"] = time.perf_counter() - t_setup
    return out


if __name__ == "__main__":
    main()
