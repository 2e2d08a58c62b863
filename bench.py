#!/usr/bin/env python
"""Benchmarks of the CCSD-gradient hot path on B200.

Default workload ``eri`` -- ERI microbenchmark, FP64 int2e_ip1 (and int2e)
over synthetic shells: 4096 shells, l in {0,1,2} (s:p:d = 4:3:2), 1-6
primitives, exponents log-uniform in [0.05, 1e4], centres in a 12-bohr cube,
seed 0; a seeded uniform sample of unique shell quartets passing a 1e-12
Schwarz screen, sorted by L-class.  One step = int2e_ip1 of every sampled
quartet, consumed in-kernel (two checksums per quartet and component).

Other workloads (``--workload``):
  lambda  Lambda/2-RDM contractions on a synthetic CCSD state (nocc 24,
          nvir 216): intermediates + 20 Jacobi Lambda updates + the 1- and
          2-particle density intermediates, once in FP64 (cuBLAS) and once in
          the split-precision tensor-core mode; errors of l1, l2 and the
          2-RDM blocks against the FP64 run.
  gemm    the split-precision tcgen05 GEMM alone (4096^3 and the vvvv-ladder
          shape 576 x 46656 x 46656) against cuBLAS DGEMM.
  grad    RHF-CCSD analytic nuclear gradient of H2O/cc-pVDZ (O at the origin,
          H at (0, +-0.757, 0.587) A): RHF + CCSD + Lambda + gradient per step,
          FP64 mode and the split-precision mode; grads/s and max|dg| between
          them; the numpy restatement of the same chain timed on the host.
  autograd  CCSDEnergy (torch.autograd.Function) forward + backward for
          ethanol/cc-pVDZ (seeded N(0, 0.02 A) displacements), FP64 and split
          precision; backward checked against central finite differences
          (1e-3 bohr, all 27 coordinates, FP64 energies).
  clusters  gradients of seeded water clusters (H2O)n, n uniform in 1..6,
          cc-pVDZ, one after another through the same chain, FP64 and split
          precision; molecules/s and per-molecule max|dg| vs FP64.

  python bench.py [--workload eri|lambda|gemm|grad|autograd|clusters] [--gpus N] [--steps K] [--warmup W]
                  [--impl ours|reference]

Multi-GPU (torchrun): every rank runs its own copy of the workload (weak
scaling, no data-path collective); time = max over ranks.
"""
import argparse
import json
import os
import sys
import threading
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# DRAM bytes per ip1 quartet of one step (warp + CTA kernels):
# dram__bytes_read.sum + dram__bytes_write.sum of both kernels in one ncu
# capture on an 8192-quartet sample of the benchmark set (cold caches; the
# Rys tables and shell data, read once per launch, are included, so the
# figure scaled to 2^18 quartets is an upper bound): (1.094 MB + 2.297 MB) / 8192
ERI_DRAM_BYTES_PER_QUARTET = (1.094e6 + 2.297e6) / 8192
METRIC = "ERI shell quartets/s (FP64 int2e_ip1, 4096 synthetic shells, Schwarz 1e-12); ERI % FP64 peak"
NSHELL = 4096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", choices=["eri", "lambda", "gemm", "grad", "autograd", "clusters", "refgpu"],
                    default="eri")
    ap.add_argument("--molecules", type=int, default=64, help="clusters workload: molecules per pass (64 = full set)")
    ap.add_argument("--serial-molecules", action="store_true",
                    help="gradient of one molecule after another instead of shape-batched solves")
    ap.add_argument("--no-molecules", action="store_true",
                    help="default workload: skip the H2O and water-cluster gradient fields")
    ap.add_argument("--no-fd", action="store_true", help="autograd workload: skip the finite-difference check")
    ap.add_argument("--polish", action="store_true",
                    help="gradient workloads: finish the split-precision T and Lambda solves with FP64 iterations "
                         "(default off: max|dg| vs FP64 is reported either way)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=None)
    ap.add_argument("--mode", default="tf32x3", help="split-precision mode of the lambda/gemm workloads")
    ap.add_argument("--nocc", type=int, default=24)
    ap.add_argument("--nvir", type=int, default=216)
    ap.add_argument("--iters", type=int, default=20, help="Lambda iterations per lambda-workload step")
    ap.add_argument("--gemm-shapes", choices=["all", "square"], default="all",
                    help="gemm workload: both shapes, or only the 4096^3 one (small, for profiling)")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--quartets", type=int, default=1 << 18, help="sampled quartets per rank per step")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample budget")
    ap.add_argument("--ref-quartets", type=int, default=4096,
                    help="reference arm: quartets of the GPU arm's list timed per step on the host")
    ap.add_argument("--no-tune", action="store_true", help="ERI workload: compiled heavy-quartet thresholds")
    args = ap.parse_args()
    dflt = {"eri": (10, 3), "lambda": (3, 3), "gemm": (10, 3), "grad": (5, 3), "autograd": (3, 3),
            "clusters": (1, 1), "refgpu": (2, 1)}[args.workload]     # clusters: one warm-up pass fills the basis caches
    args.steps = dflt[0] if args.steps is None else args.steps
    args.warmup = dflt[1] if args.warmup is None else args.warmup
    return args


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        torch.distributed.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                             timeout=datetime.timedelta(seconds=120))
    return ws, rank, local


class ClockSampler:
    """NVML sampling of SM clocks and clock-event reasons during the timed region."""

    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown",
               0x40: "hw_thermal_slowdown", 0x80: "hw_power_brake_slowdown", 0x2: "applications_clocks_setting"}

    def __init__(self, device):
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(device).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            self._h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:  # NVML missing: report that instead of guessing
            self.error = repr(e)

    def _run(self):
        nv = self._nv
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self._h, nv.NVML_CLOCK_SM))
                fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                    getattr(nv, "nvmlDeviceGetCurrentClocksThrottleReasons")
                r = fn(self._h)
                for bit, name in self.REASONS.items():
                    if r & bit:
                        self.reasons.add(name)
            except Exception:
                pass
            time.sleep(0.1)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def summary(self):
        if self._h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        return {"sm_mhz": float(np.median(self.samples)) if self.samples else None,
                "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def fp64_peak_tflops(dev):
    """Live FP64 FMA throughput (TFLOP/s), best of 5 launches."""
    from ccsd_gpu_b200 import _native
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    blocks, iters = sms * 8, 1 << 14
    out = torch.empty(blocks * 256, dtype=torch.float64, device=dev)
    best = 0.0
    for _ in range(6):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _native.call("ccsd_b200_fp64_fma_probe", _native.ptr(out), blocks, iters, _native.stream())
        b.record()
        b.synchronize()
        best = max(best, 2.0 * 8 * iters * 256 * blocks / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


def cpu_reference_rate(shells, q, deriv, budget_s):
    """Reference kernels compiled for the host (all OpenMP threads), bounded sample."""
    from oracle import eri as oeri
    kind = "reference" if oeri.ref_available() else "port"
    impl = "ref" if kind == "reference" else "oracle"
    n = min(len(q), 256)
    t = time.perf_counter()
    oeri.quartet_checksums(shells, q[:n], deriv, impl)
    dt = time.perf_counter() - t
    m = int(min(len(q), max(n, n * budget_s / max(dt, 1e-6))))
    idx = np.random.default_rng(5).permutation(len(q))[:m]
    sub = np.ascontiguousarray(q[np.sort(idx)])
    t = time.perf_counter()
    res = oeri.quartet_checksums(shells, sub, deriv, impl)
    dt = time.perf_counter() - t
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return dict(value=m / dt, unit="quartets/s", cores=threads, kind=kind,
                sample="%d of the %d sampled quartets (uniform subset), int2e_ip1, %.1f s" % (m, len(q), dt)), sub, res


def ref_list_prefix(shells, n, want, budget_s=30.0):
    """Quartets of the benchmark sample for the host-side reference runs.

    The GPU arm screens the candidate stream of workloads.sample_quartets with
    its own Schwarz kernel; here the reference's ERI kernel (compiled for the
    host) screens a prefix of the same first candidate chunk, so the quartets
    that pass are a prefix, in draw order, of the same sample: a uniform
    subset of the GPU arm's list (up to rounding of the bound at the 1e-12
    threshold).  Stops at `want` quartets or after `budget_s` of screening."""
    from oracle import eri as oeri
    impl = "ref" if oeri.ref_available() else "oracle"
    cand = workloads_mod().first_candidate_chunk(shells, n, seed=1)
    nb = shells.nbas
    qcache = {}
    kept, done = [], 0
    t0 = time.perf_counter()
    while done < len(cand) and sum(len(k) for k in kept) < want and time.perf_counter() - t0 < budget_s:
        blk = cand[done:done + 2048]
        done += len(blk)
        keys = np.concatenate([blk[:, 0].astype(np.int64) * nb + blk[:, 1], blk[:, 2].astype(np.int64) * nb + blk[:, 3]])
        new = np.unique(keys[[k not in qcache for k in keys]]) if qcache else np.unique(keys)
        if len(new):
            pr = np.stack([new // nb, new % nb], 1).astype(np.int32)
            sv = oeri.quartet_checksums(shells, np.concatenate([pr, pr], 1), 0, impl)
            for k, v in zip(new, np.sqrt(np.sqrt(np.maximum(sv[:, 0, 1], 0)))):
                qcache[int(k)] = float(v)
        qv = np.array([qcache[int(k)] for k in keys])
        kept.append(blk[qv[:len(blk)] * qv[len(blk):] > 1e-12])
    q = np.concatenate(kept, 0)[:want]
    order = np.argsort(workloads_mod().lclass(shells._bas, q), kind="stable")
    return np.ascontiguousarray(q[order]), done, time.perf_counter() - t0


def workloads_mod():
    from ccsd_gpu_b200 import workloads
    return workloads


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    from oracle import eri as oeri
    shells = workloads_mod().eri_bench_shells(NSHELL, seed=0)
    q, ncand, tscreen = ref_list_prefix(shells, args.quartets, args.ref_quartets)
    impl = "ref" if oeri.ref_available() else "oracle"
    kind = "reference" if impl == "ref" else "port"
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    times = []
    for it in range(args.warmup + args.steps):
        t = time.perf_counter()
        oeri.quartet_checksums(shells, q, 1, impl)
        dt = time.perf_counter() - t
        if it >= args.warmup:
            times.append(dt)
    v = len(q) / float(np.mean(times))
    sample = ("%d quartets: the prefix, in draw order, of the same seeded candidate stream the GPU arm screens "
              "(a uniform subset of its %d-quartet list; %d candidates screened on the host in %.1f s), "
              "int2e_ip1" % (len(q), args.quartets, ncand, tscreen))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "quartets/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(times)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "eri_microbench_4096_shells_spd_ip1", "quartets_per_step": len(q),
                       "sample_of": "the GPU arm's 2^18-quartet list (seed 1, Schwarz 1e-12)",
                       "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": threads, "kind": kind, "sample": sample},
            "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _events_timed(fn, steps, barrier, flush=None):
    """Per-step CUDA-event times (ms) on the current stream, plus the region time."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    barrier()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for a, b in evs:
        if flush is not None:
            flush.fill_(1)
        a.record()
        fn()
        b.record()
    t1.record()
    barrier()
    return np.array([a.elapsed_time(b) for a, b in evs]), t0.elapsed_time(t1)


def release_caches(dev):
    """Drop the package's device caches (captured solve graphs, packed
    split-precision operands) between workloads of one run."""
    import gc
    from ccsd_gpu_b200 import batch, contract, graphs
    batch.clear_graphs()
    graphs.clear_solve_graphs()
    contract.clear_pack_cache()
    gc.collect()
    torch.cuda.synchronize(dev)
    torch.cuda.empty_cache()


def _maxr(x, ws, dev):
    if ws == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def _tensor_peak():
    """TF32 dense peak used as the tensor roofline of the split-precision GEMMs:
    half of the measured bf16 GEMM peak (B200: TF32 runs at half the BF16 rate)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return pk["bf16_tflops"] / 2, "half of the measured bf16 burst peak (%.1f TF/s)" % pk["bf16_tflops"]
    except (OSError, KeyError, ValueError):
        return 1590.0 / 2, "half of the 1.59 PF/s bf16 fallback"


def run_gemm(args, ws, rank, local):
    """Split-precision tcgen05 GEMM vs cuBLAS DGEMM (one launch = one GEMM)."""
    from ccsd_gpu_b200.contract import STATS, check_status, contract, mark_constant, reset_stats
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    barrier = (lambda: (torch.distributed.barrier(), torch.cuda.synchronize(dev))) if ws > 1 else \
        (lambda: torch.cuda.synchronize(dev))
    g = torch.Generator(device=dev).manual_seed(rank)
    peak, peak_src = _tensor_peak()
    res = {}
    shapes = [("square_4096", 4096, 4096, 4096), ("vvvv_ladder_o24_v216", 576, 46656, 46656)]
    for name, M, N, K in shapes[:1 if args.gemm_shapes == "square" else 2]:
        a = torch.randn(M, K, dtype=torch.float64, device=dev, generator=g)
        b = torch.randn(N, K, dtype=torch.float64, device=dev, generator=g)
        mark_constant(a, b)                      # packed once; the timed region is the GEMM launch
        out = torch.empty(M, N, dtype=torch.float64, device=dev)
        run = lambda: contract("mk,nk->mn", a, b, out=out, mode=args.mode)   # noqa: E731
        for _ in range(args.warmup):
            run()
        reset_stats()
        with ClockSampler(dev) as clk:
            ks, _ = _events_timed(run, args.steps, barrier)
        launches = STATS["launches"]
        check_status(dev)
        ms = _maxr(float(ks.mean()), ws, dev)
        ref = a @ b.T
        err = float((out - ref).abs().max() / ref.abs().max())
        dg = lambda: torch.mm(a, b.T, out=ref)   # noqa: E731
        dg()
        kd, _ = _events_timed(dg, max(3, args.steps // 2), barrier)
        ms_d = _maxr(float(kd.mean()), ws, dev)
        fl = 2.0 * M * N * K
        res[name] = {"ms": ms, "fp64_equiv_tflops": fl / ms / 1e9, "tensor_tflops": 3 * fl / ms / 1e9,
                     "dgemm_ms": ms_d, "dgemm_tflops": fl / ms_d / 1e9, "speedup_vs_dgemm": ms_d / ms,
                     "max_rel_err_vs_dgemm": err, "launches_timed": launches, "clocks": clk.summary()}
        del a, b, out, ref
        torch.cuda.empty_cache()
    head = res[list(res)[-1]]
    line = {"metric": "split-precision GEMM FP64-equivalent TFLOP/s (%s, vvvv-ladder shape)" % args.mode,
            "value": head["fp64_equiv_tflops"] * ws, "unit": "TFLOP/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.mode, "data": "synthetic",
            "config": {"workload": "tc_split_gemm", "headline_shape": list(res)[-1], "shapes": res,
                       "l2": "operands larger than L2 (vvvv shape: 17.4 GB B operand)",
                       "parallelism": "dp%d" % ws if ws > 1 else "single"},
            "roofline": {"bound": "tensor", "achieved": head["tensor_tflops"], "peak": peak, "unit": "TFLOP/s",
                         "frac": head["tensor_tflops"] / peak, "traffic": None,
                         "peak_source": peak_src, "flops": "3 TF32 products x 2 M N K per GEMM"},
            "gpu_launches": head["launches_timed"], "clocks": head["clocks"], "cpu_baseline": None,
            "e2e": None}
    if rank == 0:
        print(json.dumps(line), flush=True)


def _rel(a, b):
    d = float((a - b).abs().max())
    m = float(b.abs().max())
    return d / m if m > 0 else d


def _lambda_solver(t1, t2, deris, iters, keep):
    from types import SimpleNamespace
    from ccsd_gpu_b200.gpu_ccsd_grad import _gamma1_intermediates_gpu, _gamma2_intermediates_gpu
    from ccsd_gpu_b200.gpu_ccsd_lambda import make_intermediates_gpu, update_lambda_gpu

    def solve(mode):
        cc = SimpleNamespace(level_shift=0.0, precision=mode)
        imds = make_intermediates_gpu(cc, t1, t2, deris, mode)
        l1, l2 = t1, t2
        for _ in range(iters):
            l1, l2 = update_lambda_gpu(cc, t1, t2, l1, l2, deris, imds, mode=mode)
        d1 = _gamma1_intermediates_gpu(cc, t1, t2, l1, l2)
        d2 = _gamma2_intermediates_gpu(cc, t1, t2, l1, l2)
        # copies: the compared results must not share storage that a later
        # solve (of either mode) writes into
        cp = lambda x: x.clone() if x is not None else None      # noqa: E731
        keep[mode] = (cp(l1), cp(l2), tuple(cp(x) for x in d1), tuple(cp(x) for x in d2))
    return solve


def lambda_cpu_baseline(args, dev, full_flops, nocc=16, nvir=144):
    """The oracle's numpy restatement of the reference's Lambda/RDM path
    (oracle/cc_oracle.py: make_intermediates, update_lambda, gamma1, gamma2, the
    equations of ref: ccsd_gpu/gpu_ccsd_lambda.py:68-337 and
    ccsd_gpu/gpu_ccsd_grad.py:101-246) on the host cores, on a bounded sample:
    the same synthetic state at (nocc, nvir) = (16, 144), intermediates + two
    timed Lambda iterations (times iterations) + the RDM intermediates.  Scaled
    to the benchmark's size by the ratio of counted contraction flops of the
    package's FP64 run at the two sizes (the full-size numpy run needs tens of
    GB of host temporaries)."""
    from types import SimpleNamespace
    from oracle import cc_oracle
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.contract import STATS, reset_stats
    from ccsd_gpu_b200.gpu_ccsd_lambda import DeviceEris
    eris, t1, t2 = workloads.lambda_bench_state(nocc, nvir, seed=0, device=dev)
    h = lambda x: x.detach().cpu().numpy()      # noqa: E731
    E = SimpleNamespace(**{k: h(getattr(eris, k)) for k in ("oooo", "ovoo", "ovvo", "oovv", "ovov", "ovvv", "vvvv")})
    fock, moe, t1h, t2h = h(eris.fock), h(eris.mo_energy), h(t1), h(t2)
    # counted flops of the same run at the sample size (package, FP64)
    deris = DeviceEris(eris, dev)
    keep = {}
    solve = _lambda_solver(t1, t2, deris, args.iters, keep)
    reset_stats()
    solve("fp64")
    torch.cuda.synchronize(dev)
    small_flops = STATS["flops"]
    del deris, keep, eris
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    imds = cc_oracle.make_intermediates(t1h, t2h, fock, E)
    t_imd = time.perf_counter() - t0
    l1, l2 = t1h, t2h
    n_it = 2
    t0 = time.perf_counter()
    for _ in range(n_it):
        l1, l2 = cc_oracle.update_lambda(t1h, t2h, l1, l2, fock, moe, E, imds)
    t_it = (time.perf_counter() - t0) / n_it
    t0 = time.perf_counter()
    cc_oracle.gamma1(t1h, t2h, l1, l2)
    cc_oracle.gamma2(t1h, t2h, l1, l2)
    t_rdm = time.perf_counter() - t0
    t_small = t_imd + args.iters * t_it + t_rdm
    scale = full_flops / small_flops
    return {"value": t_small * scale, "unit": "s/run", "cores": os.cpu_count(), "kind": "port",
            "sample": "numpy oracle at nocc %d, nvir %d: intermediates %.2f s + %d x %.2f s per Lambda iteration "
                      "(2 timed) + RDM %.2f s = %.1f s, scaled x%.1f by counted contraction flops to nocc %d, "
                      "nvir %d" % (nocc, nvir, t_imd, args.iters, t_it, t_rdm, t_small, scale, args.nocc, args.nvir)}


def measure_lambda(args, ws, rank, dev, steps, warmup, cpu=False):
    """Configuration 3: intermediates + iters Lambda updates + RDM intermediates
    of the synthetic (nocc, nvir) state, FP64 and the split mode (dict)."""
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.contract import STATS, check_status, reset_stats
    from ccsd_gpu_b200.gpu_ccsd_lambda import DeviceEris
    barrier = _barrier_fn(ws, dev)
    eris, t1, t2 = workloads.lambda_bench_state(args.nocc, args.nvir, seed=rank, device=dev)
    deris = DeviceEris(eris, dev)
    del eris
    keep = {}
    solve = _lambda_solver(t1, t2, deris, args.iters, keep)
    out = {}
    for mode in ("fp64", args.mode):
        keep.pop(mode, None)
        for _ in range(warmup):
            solve(mode)
        reset_stats()
        with ClockSampler(dev) as clk:
            ks, region = _events_timed(lambda: solve(mode), steps, barrier)
        check_status(dev)
        out[mode] = {"s_per_run": _maxr(float(ks.mean()), ws, dev) * 1e-3, "flops": STATS["flops"] / steps,
                     "launches": STATS["launches"] // steps, "clocks": clk.summary()}
        if mode != "fp64":
            ref, got = keep["fp64"], keep[mode]
            d2e = max(_rel(x, y) for x, y in zip(got[3], ref[3]) if x is not None)
            d1e = max(_rel(x, y) for x, y in zip(got[2], ref[2]))
            out[mode].update(l1_rel_err=_rel(got[0], ref[0]), l2_rel_err=_rel(got[1], ref[1]),
                             rdm1_rel_err=d1e, rdm2_rel_err=d2e)
            del keep["fp64"]
        torch.cuda.empty_cache()
    del deris, keep, t1, t2
    torch.cuda.empty_cache()
    fp, mx = out["fp64"], out[args.mode]
    peak, peak_src = _tensor_peak()
    ach = 3 * mx["flops"] / mx["s_per_run"] / 1e12
    res = {"workload": "lambda_rdm_o%d_v%d" % (args.nocc, args.nvir), "iterations": args.iters,
           "steps": steps, "warmup": warmup, "fp64": fp, "mixed": mx,
           "speedup_vs_fp64": fp["s_per_run"] / mx["s_per_run"],
           "roofline": {"bound": "tensor", "achieved": ach, "peak": peak, "unit": "TFLOP/s", "frac": ach / peak,
                        "traffic": None, "peak_source": peak_src,
                        "flops": "3 TF32 products x counted 2 M N K of every contraction in the run"},
           "cpu_baseline": None}
    if cpu and rank == 0:
        res["cpu_baseline"] = lambda_cpu_baseline(args, dev, fp["flops"])
    return res


def run_lambda(args, ws, rank, local):
    """Lambda/2-RDM contraction bench on a synthetic CCSD state."""
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = measure_lambda(args, ws, rank, dev, args.steps, args.warmup, cpu=True)
    mx = r["mixed"]
    line = {"metric": "Lambda/2-RDM run time (nocc %d, nvir %d, %d Lambda iterations + RDM intermediates), %s vs FP64"
                      % (args.nocc, args.nvir, args.iters, args.mode),
            "value": mx["s_per_run"], "unit": "s/run", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": mx["s_per_run"] * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": args.mode, "data": "synthetic",
            "config": {"workload": r["workload"], "iterations": args.iters,
                       "state": "seeded synthetic CCSD state (lambda_bench_state)",
                       "l2": "operands larger than L2 (vvvv block 17.4 GB)",
                       "parallelism": "dp%d" % ws if ws > 1 else "single"},
            "fp64": r["fp64"], "mixed": mx, "speedup_vs_fp64": r["speedup_vs_fp64"], "roofline": r["roofline"],
            "gpu_launches": mx["launches"], "clocks": mx["clocks"], "cpu_baseline": r["cpu_baseline"], "e2e": None}
    if rank == 0:
        print(json.dumps(line), flush=True)


H2O_CCPVDZ = "O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587"


def _barrier_fn(ws, dev):
    return (lambda: (torch.distributed.barrier(), torch.cuda.synchronize(dev))) if ws > 1 else \
        (lambda: torch.cuda.synchronize(dev))


def measure_h2o(args, ws, rank, dev, steps, warmup, cpu=True):
    """Configuration 1: RHF + CCSD + Lambda + gradient of H2O/cc-pVDZ per step,
    FP64 mode and the split-precision mode (dict of results)."""
    from ccsd_gpu_b200 import _native
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.gto import M
    from ccsd_gpu_b200.scf import RHF
    barrier = _barrier_fn(ws, dev)
    mol = M(atom=H2O_CCPVDZ, basis="cc-pvdz")
    grads = {}

    def step(mode):
        def run():
            cc = CCSD(RHF(mol).run(), precision=mode)
            cc.t_polish = cc.lambda_polish = args.polish
            cc.kernel()
            cc.conv_tol_normt = 1e-9
            grads[mode] = cc.nuc_grad_method().kernel()        # numpy (natm, 3): the D2H read
        return run

    res = {}
    for mode in ("fp64", args.mode):
        fn = step(mode)
        for _ in range(warmup):
            fn()
        n0 = sum(_native.CALLS.values())
        with ClockSampler(dev) as clk:
            ks, _ = _events_timed(fn, steps, barrier)
        res[mode] = {"s_per_grad": _maxr(float(ks.mean()), ws, dev) * 1e-3, "clocks": clk.summary(),
                     "launches": (sum(_native.CALLS.values()) - n0) // steps}
    out = {"workload": "h2o_ccpvdz_ccsd_gradient", "nao": mol.nao_nr(), "nocc": mol.nelectron // 2,
           "steps": steps, "warmup": warmup,
           "fp64_grads_per_s": ws / res["fp64"]["s_per_grad"], "mixed_grads_per_s": ws / res[args.mode]["s_per_grad"],
           "speedup_vs_fp64": res["fp64"]["s_per_grad"] / res[args.mode]["s_per_grad"],
           "max_abs_dg_vs_fp64": float(np.abs(grads[args.mode] - grads["fp64"]).max()),
           "mixed": res[args.mode], "fp64": res["fp64"], "cpu_baseline": None,
           "h2d_bytes_per_step": int(mol._atm.nbytes + mol._env.nbytes + mol._bas.nbytes),
           "d2h_bytes_per_step": int(grads[args.mode].nbytes)}
    if cpu and rank == 0 and ws == 1:
        from oracle import scf_cc_oracle as Q
        t = time.perf_counter()
        _, g_ref = Q.ccsd_gradient(mol)
        dt = time.perf_counter() - t
        out["cpu_baseline"] = {
            "value": 1.0 / dt, "unit": "grads/s", "cores": int(torch.get_num_threads()), "kind": "port",
            "sample": "one H2O/cc-pVDZ CCSD gradient by the numpy restatement of the chain (%.1f s)" % dt,
            "max_abs_dg_fp64_gpu_vs_port": float(np.abs(grads["fp64"] - g_ref).max())}
    return out


def run_grad(args, ws, rank, local):
    """Full CCSD gradient of H2O/cc-pVDZ per step, FP64 vs split precision."""
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = measure_h2o(args, ws, rank, dev, args.steps, args.warmup)
    mx = r["mixed"]
    line = {"metric": "CCSD grads/s, H2O/cc-pVDZ (RHF + CCSD + Lambda + gradient per step), %s vs FP64" % args.mode,
            "value": r["mixed_grads_per_s"], "unit": "grads/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mx["s_per_grad"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.mode, "data": "synthetic",
            "config": {"workload": r["workload"], "fp64_polish": args.polish, "nao": r["nao"], "nocc": r["nocc"],
                       "l2": "latency-bound chain; no flush",
                       "parallelism": "dp%d" % ws if ws > 1 else "single"},
            "fp64_grads_per_s": r["fp64_grads_per_s"], "mixed_grads_per_s": r["mixed_grads_per_s"],
            "speedup_vs_fp64": r["speedup_vs_fp64"], "max_abs_dg_vs_fp64": r["max_abs_dg_vs_fp64"],
            "roofline": None, "gpu_launches": mx["launches"], "clocks": mx["clocks"], "cpu_baseline": r["cpu_baseline"],
            "e2e": {"value": r["mixed_grads_per_s"], "unit": "grads/s", "h2d_bytes_per_step": r["h2d_bytes_per_step"],
                    "d2h_bytes_per_step": r["d2h_bytes_per_step"]}}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_refgpu(args, ws, rank, local):
    """Reference-GPU comparator: int2e_ip1 (and int2e) Cartesian s2kl blocks of
    every atom's shells, as the reference's gradient loop requests them
    (ref: ccsd_gpu/gpu_ccsd_grad.py:449-457), from the package's kernels and from
    the reference's own kernels built for sm_100a and launched by its launch loop
    (oracle/_ref/libref_eri_gpu.so; a baseline leg, never the product path).
    Also times the package's fused ip1-Gamma gradient contraction of the whole
    molecule, which replaces the blocks in the package's gradient."""
    from oracle import ref_gpu
    from ccsd_gpu_b200 import compute_int2e_gpu, compute_int2e_ip1_gpu, workloads
    from ccsd_gpu_b200.cuda.ip1_contract import contract_int2e_ip1
    from ccsd_gpu_b200.gto import M
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if not ref_gpu.available():
        if rank == 0:
            print(json.dumps({"workload": "refgpu", "unavailable": "oracle/_ref/libref_eri_gpu.so not built"}))
        return
    barrier = (lambda: (torch.distributed.barrier(), torch.cuda.synchronize(dev))) if ws > 1 else \
        (lambda: torch.cuda.synchronize(dev))
    sym, xyz = workloads.ethanol_atoms(seed=0)
    mols = {"h2o": "O 0 0 0; H 0 0.757 0.587; H 0 -0.757 0.587",
            "ethanol": workloads.atom_string(sym, xyz)}
    rng = np.random.default_rng(0)
    for n in (6,):
        s6, x6 = workloads.water_cluster_atoms(n, rng)
        mols["h2o_6"] = workloads.atom_string(s6, x6)
    out = {}
    steps = max(1, min(args.steps, 3))
    for name, atom in mols.items():
        mol = M(atom=atom, basis="cc-pvdz", cart=True)
        rb = ref_gpu.RefBasis(mol, dev)
        blocks = [(int(r[0]), int(r[1])) for r in mol.offset_nr_by_atom()]
        res = {"nao_cart": int(mol.nao_nr()), "atom_blocks": len(blocks)}
        for deriv in (1, 0):
            fn = compute_int2e_ip1_gpu if deriv else compute_int2e_gpu
            worst = 0.0
            for b0, b1 in blocks:       # parity (and warm-up) on every block
                ref = ref_gpu.eri_cart(rb, b0, b1, deriv)
                got = fn(mol, b0, b1)
                err = float((got - ref).abs().max() / (ref.abs().max() + 1e-300))
                worst = max(worst, err)
                del ref, got
            torch.cuda.empty_cache()

            def run_ref():
                for b0, b1 in blocks:
                    ref_gpu.eri_cart(rb, b0, b1, deriv)

            def run_ours():
                for b0, b1 in blocks:
                    fn(mol, b0, b1)
            with ClockSampler(dev) as clk:
                kr, _ = _events_timed(run_ref, steps, barrier)
                ko, _ = _events_timed(run_ours, steps, barrier)
            tr, to = _maxr(float(kr.mean()), ws, dev), _maxr(float(ko.mean()), ws, dev)
            res["ip1" if deriv else "int2e"] = {
                "reference_kernels_ms": tr, "package_kernels_ms": to, "speedup": tr / to,
                "max_rel_diff_vs_reference_kernels": worst, "clocks": clk.summary()}
        msph = M(atom=atom, basis="cc-pvdz")
        nao = msph.nao_nr()
        g = torch.randn((nao,) * 4, dtype=torch.float64, device=dev, generator=torch.Generator(dev).manual_seed(0))
        g = g + g.transpose(2, 3)
        contract_int2e_ip1(msph, g)
        kf, _ = _events_timed(lambda: contract_int2e_ip1(msph, g), steps, barrier)
        res["fused_ip1_gamma_ms"] = _maxr(float(kf.mean()), ws, dev)
        res["fused_speedup_vs_reference_ip1_blocks"] = res["ip1"]["reference_kernels_ms"] / res["fused_ip1_gamma_ms"]
        del g
        torch.cuda.empty_cache()
        out[name] = res
    big = out["h2o_6"]["ip1"]
    line = {"metric": "int2e_ip1 atom-block time, reference's kernels / package's kernels on the same B200",
            "value": big["speedup"], "unit": "x", "n_gpus": ws, "steps": steps, "warmup": 1,
            "ms_per_step": big["package_kernels_ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic geometries",
            "config": {"workload": "eri_atom_blocks_refgpu", "basis": "cc-pvdz (Cartesian blocks)",
                       "value_of": "(H2O)6 int2e_ip1",
                       "reference_launch": "one launch per decontracted i-shell, dim3(1, 32) blocks, as "
                                           "ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216",
                       "parallelism": "dp%d" % ws if ws > 1 else "single"},
            "molecules": out, "roofline": None, "cpu_baseline": None, "e2e": None}
    if rank == 0:
        print(json.dumps(line), flush=True)


def _ccsd_energy(mol, mode):
    from ccsd_gpu_b200.ccsd import CCSD
    from ccsd_gpu_b200.scf import RHF
    cc = CCSD(RHF(mol).run(), precision=mode)
    cc.kernel()
    return cc.e_tot


def measure_autograd(args, ws, rank, dev, steps, warmup, fd=True):
    """Configuration 4: CCSDEnergy forward + backward for ethanol/cc-pVDZ, FP64
    and the split mode, and a central-FD check of the backward (dict)."""
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.gpu_ccsd_grad import CCSDEnergy
    from ccsd_gpu_b200.gto import M
    barrier = _barrier_fn(ws, dev)
    sym, xyz = workloads.ethanol_atoms(seed=0)
    mol = M(atom=workloads.atom_string(sym, xyz), basis="cc-pvdz")
    x0 = torch.tensor(mol.atom_coords(), dtype=torch.float64)
    grads = {}

    def step(mode):
        def run():
            x = x0.to(dev).requires_grad_(True)
            e = CCSDEnergy.apply(x, mol, mode, 0, args.polish)
            e.backward()
            grads[mode] = x.grad.detach().cpu().numpy()
        return run

    res = {}
    for mode in ("fp64", args.mode):
        fn = step(mode)
        for _ in range(warmup):
            fn()
        with ClockSampler(dev) as clk:
            ks, _ = _events_timed(fn, steps, barrier)
        res[mode] = {"s_per_grad": _maxr(float(ks.mean()), ws, dev) * 1e-3, "clocks": clk.summary()}
    fd_err = None
    if fd and rank == 0:
        h = 1e-3
        fdg = np.zeros_like(grads["fp64"])
        for a in range(mol.natm):
            for c in range(3):
                ep = []
                for sgn in (1, -1):
                    xs = x0.numpy().copy()
                    xs[a, c] += sgn * h
                    ep.append(_ccsd_energy(mol.copy().set_geom_(xs), "fp64"))
                fdg[a, c] = (ep[0] - ep[1]) / (2 * h)
        fd_err = {"max_abs_fd_minus_fp64_backward": float(np.abs(fdg - grads["fp64"]).max()),
                  "max_abs_fd_minus_mixed_backward": float(np.abs(fdg - grads[args.mode]).max()),
                  "step_bohr": h, "coordinates": int(fdg.size)}
    return {"workload": "ethanol_ccpvdz_autograd", "nao": mol.nao_nr(), "nocc": mol.nelectron // 2,
            "steps": steps, "warmup": warmup,
            "fp64_grads_per_s": ws / res["fp64"]["s_per_grad"], "mixed_grads_per_s": ws / res[args.mode]["s_per_grad"],
            "speedup_vs_fp64": res["fp64"]["s_per_grad"] / res[args.mode]["s_per_grad"],
            "max_abs_dg_vs_fp64": float(np.abs(grads[args.mode] - grads["fp64"]).max()),
            "finite_difference": fd_err, "fp64": res["fp64"], "mixed": res[args.mode]}


def run_autograd(args, ws, rank, local):
    """CCSDEnergy forward + backward for ethanol/cc-pVDZ; central-FD check."""
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = measure_autograd(args, ws, rank, dev, args.steps, args.warmup, fd=not args.no_fd)
    mx = r["mixed"]
    line = {"metric": "CCSDEnergy forward+backward per s, ethanol/cc-pVDZ, %s vs FP64" % args.mode,
            "value": r["mixed_grads_per_s"], "unit": "grads/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": mx["s_per_grad"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": args.mode, "data": "synthetic",
            "config": {"workload": r["workload"], "fp64_polish": args.polish, "nao": r["nao"], "nocc": r["nocc"],
                       "geometry": "standard internal coordinates + N(0, 0.02 A) displacements, seed 0",
                       "parallelism": "dp%d" % ws if ws > 1 else "single"},
            "fp64_grads_per_s": r["fp64_grads_per_s"], "mixed_grads_per_s": r["mixed_grads_per_s"],
            "speedup_vs_fp64": r["speedup_vs_fp64"], "max_abs_dg_vs_fp64": r["max_abs_dg_vs_fp64"],
            "finite_difference": r["finite_difference"], "roofline": None, "clocks": mx["clocks"],
            "cpu_baseline": None, "e2e": None}
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_clusters(args, ws, rank, dev, nmol, dropin=False):
    """Configuration 5: gradients of the seeded (H2O)n clusters (n in 1..6),
    FP64 mode and the split-precision mode.  Rank r takes clusters r, r + N,
    ... of the first nmol.  One warm-up pass over one cluster of each size
    fills the basis, tuning and graph caches; then one timed pass per mode."""
    from ccsd_gpu_b200 import batch, workloads
    from ccsd_gpu_b200.gto import M
    barrier = _barrier_fn(ws, dev)
    allc = workloads.water_clusters(64, seed=0)
    mine = [allc[i % 64] for i in range(rank, nmol, ws)]
    mols = [M(atom=workloads.atom_string(s, x), basis="cc-pvdz") for s, x in mine]
    warm, seen = [], set()
    for m in mols:
        if m.natm not in seen:
            seen.add(m.natm)
            warm.append(m)
    grads, res = {}, {}
    for mode in ("fp64", args.mode):
        batch.gradients(warm, mode, polish=args.polish, batched=not args.serial_molecules)
        with ClockSampler(dev) as clk:
            barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            grads[mode] = batch.gradients(mols, mode, polish=args.polish, batched=not args.serial_molecules)
            b.record()
            barrier()
        res[mode] = {"s_per_pass": _maxr(a.elapsed_time(b) * 1e-3, ws, dev), "clocks": clk.summary()}
    if dropin:
        # the plain FP64 drop-in path: one molecule after another through the
        # FP64 chain (no shape batching), as the reference runs one molecule
        batch.gradients(warm, "fp64", polish=args.polish, batched=False)
        with ClockSampler(dev) as clk:
            barrier()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            gd = batch.gradients(mols, "fp64", polish=args.polish, batched=False)
            b.record()
            barrier()
        res["fp64_dropin"] = {"s_per_pass": _maxr(a.elapsed_time(b) * 1e-3, ws, dev), "clocks": clk.summary(),
                              "max_abs_dg_vs_batched_fp64": max(float(np.abs(x - y).max())
                                                                for x, y in zip(gd, grads["fp64"]))}
    dg = [float(np.abs(x - y).max()) for x, y in zip(grads[args.mode], grads["fp64"])]
    total = len(allc[:nmol]) if nmol <= 64 else nmol
    return {"workload": "water_clusters_ccpvdz", "molecules": total, "molecules_per_rank": len(mols),
            "waters_per_molecule": [m.natm // 3 for m in mols],
            "batched": not args.serial_molecules, "fp64_polish": args.polish,
            "fp64_molecules_per_s": total / res["fp64"]["s_per_pass"],
            "mixed_molecules_per_s": total / res[args.mode]["s_per_pass"],
            "speedup_vs_fp64": res["fp64"]["s_per_pass"] / res[args.mode]["s_per_pass"],
            "per_molecule_max_abs_dg_vs_fp64": dg, "max_abs_dg_vs_fp64": max(dg),
            "fp64": res["fp64"], "mixed": res[args.mode],
            "fp64_dropin": res.get("fp64_dropin"),
            "fp64_dropin_molecules_per_s": total / res["fp64_dropin"]["s_per_pass"] if dropin else None,
            "speedup_vs_fp64_dropin": (res["fp64_dropin"]["s_per_pass"] / res[args.mode]["s_per_pass"]
                                       if dropin else None)}


def run_clusters(args, ws, rank, local):
    """Gradients of seeded water clusters, FP64 and split precision."""
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    r = measure_clusters(args, ws, rank, dev, args.molecules, dropin=True)
    mx = r["mixed"]
    line = {"metric": "CCSD gradients of (H2O)n clusters, n in 1..6, cc-pVDZ: molecules/s, %s vs FP64" % args.mode,
            "value": r["mixed_molecules_per_s"], "unit": "molecules/s", "n_gpus": ws,
            "steps": 1, "warmup": 1, "ms_per_step": mx["s_per_pass"] * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": args.mode,
            "data": "synthetic",
            "config": {"workload": r["workload"], "fp64_polish": args.polish, "molecules": r["molecules"],
                       "batched": r["batched"], "waters_per_molecule": r["waters_per_molecule"],
                       "cluster_set": "64 seeded clusters (seed 0), first %d" % r["molecules"],
                       "parallelism": "dp%d" % ws if ws > 1 else "single"},
            "fp64_molecules_per_s": r["fp64_molecules_per_s"], "mixed_molecules_per_s": r["mixed_molecules_per_s"],
            "speedup_vs_fp64": r["speedup_vs_fp64"],
            "fp64_dropin_molecules_per_s": r["fp64_dropin_molecules_per_s"],
            "speedup_vs_fp64_dropin": r["speedup_vs_fp64_dropin"],
            "per_molecule_max_abs_dg_vs_fp64": r["per_molecule_max_abs_dg_vs_fp64"],
            "max_abs_dg_vs_fp64": r["max_abs_dg_vs_fp64"],
            "roofline": None, "clocks": mx["clocks"], "cpu_baseline": None, "e2e": None}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
        if ws > 1:
            torch.distributed.destroy_process_group()
        return
    if args.workload != "eri":
        {"gemm": run_gemm, "lambda": run_lambda, "grad": run_grad, "autograd": run_autograd,
         "clusters": run_clusters, "refgpu": run_refgpu}[args.workload](args, ws, rank, local)
        if ws > 1:
            torch.distributed.destroy_process_group()
        return
    from ccsd_gpu_b200 import workloads
    from ccsd_gpu_b200.cuda.quartets import DeviceShells, quartet_checksums, schwarz_bounds
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    shells = workloads.eri_bench_shells(NSHELL, seed=0)
    ds = DeviceShells(shells, dev)
    q = workloads.sample_quartets(shells, args.quartets, seed=1 + rank, schwarz_fn=lambda p: schwarz_bounds(ds, p))
    nq = len(q)
    flops_ip1 = workloads.quartet_flops(shells, q, 1)
    flops_int2e = workloads.quartet_flops(shells, q, 0)
    flops_ip1_all = workloads.quartet_flops(shells, q, 1, screened=False)
    classes, counts = np.unique(workloads.lclass(shells._bas, q), return_counts=True)
    peak = fp64_peak_tflops(dev)

    q_host = torch.from_numpy(q).pin_memory()
    q_dev = q_host.to(dev)
    out = torch.empty((nq, 3, 2), dtype=torch.float64, device=dev)
    out0 = torch.empty((nq, 1, 2), dtype=torch.float64, device=dev)
    out_host = torch.empty((nq, 3, 2), dtype=torch.float64).pin_memory()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # 256 MiB > 126 MB L2
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    def timed(fn, steps):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for a, b in evs:
            flush.fill_(1)
            a.record()
            fn()
            b.record()
        t1.record()
        barrier()
        return np.array([a.elapsed_time(b) for a, b in evs]), t0.elapsed_time(t1)

    # autotuner (before warm-up, outside every timed region): heavy-quartet
    # threshold of each derivative order for this list's class mix
    from ccsd_gpu_b200 import tune
    tune.enable(not args.no_tune)
    dshare = float((shells._bas[:, 1][q].max(1) >= 2).mean())
    heavy = {d: tune.tune_eri_heavy(ds, shells._bas, q_dev, d, dshare) for d in (1, 0)}
    paths = {d: tune.tune_eri_paths(ds, shells._bas, q_dev, d, dshare) for d in (1, 0)}
    ip1 = lambda: quartet_checksums(ds, q_dev, 1, out=out)   # noqa: E731
    for _ in range(args.warmup):
        ip1()
    torch.cuda.synchronize(dev)
    with ClockSampler(dev) as clk:
        ks, region_ms = timed(ip1, args.steps)
    kernel_ms = float(ks.mean())

    def maxr(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    kernel_ms_max = maxr(kernel_ms)
    # int2e on the same sample (reported beside the headline)
    i2 = lambda: quartet_checksums(ds, q_dev, 0, out=out0)   # noqa: E731
    i2()
    ks0, _ = timed(i2, max(3, args.steps // 2))
    int2e_ms = maxr(float(ks0.mean()))

    # end to end through the public API: pinned host quartets in, checksums out
    def e2e_step():
        q_dev.copy_(q_host, non_blocking=True)
        quartet_checksums(ds, q_dev, 1, out=out)
        out_host.copy_(out, non_blocking=True)
    e2e_step()
    ke, _ = timed(e2e_step, args.steps)
    e2e_ms = maxr(float(ke.mean()))

    cpu = None
    parity = None
    if rank == 0 and ws == 1:
        cpu, sub, ref_vals = cpu_reference_rate(shells, q, 1, args.cpu_seconds)
        # parity of the measured kernel against the reference build on the CPU
        # subset: the weighted checksum s1 = sum_f w_f I_f (w in [1, 1.875]) of
        # each quartet and component; |ds1| <= 1e-10 * 2 sqrt(nf sum I^2) +
        # 2e-12 nf is the 1e-10 elementwise bar with a small absolute floor
        gsub = quartet_checksums(ds, torch.from_numpy(sub).to(dev), 1).cpu().numpy()
        l = shells._bas[:, 1][sub]
        nf = np.prod((l + 1) * (l + 2) // 2, axis=1)[:, None].astype(np.float64)
        scale = 2 * np.sqrt(nf * np.abs(ref_vals[..., 1]))
        diff = np.abs(gsub[..., 0] - ref_vals[..., 0])
        rel_ok = scale > 100 * 2e-12 * nf          # not dominated by the absolute floor
        parity = {"checksums_close": bool((diff <= 1e-10 * scale + 2e-12 * nf).all()),
                  "max_rel_err": float((diff[rel_ok] / scale[rel_ok]).max()) if rel_ok.any() else None,
                  "max_abs_err": float(diff.max()), "quartets": int(len(sub)),
                  "rel_err_over": "quartets whose checksum scale exceeds 100x the absolute floor"}

    tot_q = nq * ws
    value = tot_q / (kernel_ms_max * 1e-3)
    achieved = flops_ip1 / (kernel_ms * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kernel_ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "eri_microbench_4096_shells_spd_ip1", "nshell": NSHELL, "quartets_per_rank": nq,
                   "lclasses": int(len(classes)), "schwarz": 1e-12,
                   "heavy_nf": {"int2e": heavy[0], "ip1": heavy[1], "autotuned": not args.no_tune},
                   "paths": {("int2e", "ip1")[d]: {"contracted_hrr": paths[d].count(1),
                                                   "per_output": paths[d].count(2),
                                                   "compiled_rule": paths[d].count(0)} for d in (0, 1)},
                   "l2": "256 MiB buffer written between steps, outside the per-step kernel events",
                   "parallelism": "dp%d" % ws if ws > 1 else "single"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": ERI_DRAM_BYTES_PER_QUARTET * nq,
                     "traffic_source": "DRAM bytes (read + write) of one ncu capture of the ip1 warp and CTA "
                                       "kernels on an 8192-quartet sample of this set, scaled per quartet; an "
                                       "upper bound (per-launch table and shell reads are included)",
                     "peak_source": "FP64 FMA probe measured in this run (driver peaks file has no FP64 figure)",
                     "flops": "reference-algorithm FP64 op count of the primitive quartets of the sample that "
                              "pass the primitive-pair screen (the ones the kernels evaluate)",
                     "unscreened_equivalent_frac": flops_ip1_all / (kernel_ms * 1e-3) / 1e12 / peak},
        "int2e_quartets_per_s": tot_q / (int2e_ms * 1e-3),
        "int2e_roofline_frac": flops_int2e / (int2e_ms * 1e-3) / 1e12 / peak,
        "timed_region_ms": region_ms,
        "e2e": {"value": tot_q / (e2e_ms * 1e-3), "unit": "quartets/s", "h2d_bytes_per_step": nq * 16,
                "d2h_bytes_per_step": nq * 3 * 2 * 8},
        "gpu_launches": 2 * args.steps,     # per step: the warp-per-quartet and the CTA (heavy) kernel
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "parity_vs_reference": parity,
    }
    if not args.no_molecules:
        # the metric's other clauses, measured after (outside) the ERI timed
        # region: configuration 1 (H2O/cc-pVDZ gradient), configuration 5 (the
        # 64 seeded water clusters), configuration 4 (ethanol CCSDEnergy forward
        # + backward, FD-checked) and, from released caches, configuration 3
        # (Lambda/RDM contractions, nocc 24, nvir 216); FP64 mode against the
        # split-precision mode
        h2o = measure_h2o(args, ws, rank, dev, steps=10, warmup=3)
        for k in ("mixed", "fp64"):
            h2o[k].pop("clocks", None)
        line["h2o_ccpvdz_gradient"] = h2o
        cl = measure_clusters(args, ws, rank, dev, 64, dropin=True)
        line["water_clusters_gradient"] = cl
        line["ethanol_ccpvdz_autograd"] = measure_autograd(args, ws, rank, dev, steps=2, warmup=1, fd=True)
        release_caches(dev)
        line["lambda_rdm"] = measure_lambda(args, ws, rank, dev, steps=1, warmup=1, cpu=False)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
