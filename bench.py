#!/usr/bin/env python
"""ERI microbenchmark on B200: FP64 int2e_ip1 (and int2e) over synthetic shells.

Workload: 4096 shells, l in {0,1,2} (s:p:d = 4:3:2), 1-6 primitives,
exponents log-uniform in [0.05, 1e4], centres in a 12-bohr cube, seed 0; a
seeded uniform sample of unique shell quartets passing a 1e-12 Schwarz
screen, sorted by L-class.  One step = int2e_ip1 of every sampled quartet,
consumed in-kernel (two checksums per quartet and component).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank draws its own sample (weak scaling, no
data-path collective); time = max over ranks.
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

METRIC = "ERI shell quartets/s (FP64 int2e_ip1, 4096 synthetic shells, Schwarz 1e-12); ERI % FP64 peak"
NSHELL = 4096


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--quartets", type=int, default=1 << 18, help="sampled quartets per rank per step")
    ap.add_argument("--cpu-seconds", type=float, default=10.0, help="CPU-baseline sample budget")
    return ap.parse_args()


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


def run_reference_arm(args, ws, rank):
    if rank != 0:
        return
    from ccsd_gpu_b200 import workloads
    from oracle import eri as oeri
    shells = workloads.eri_bench_shells(NSHELL, seed=0)
    # Schwarz bounds on the host with the same screen (Frobenius bound of (ij|ij))
    def qfn(pairs):
        s = oeri.quartet_checksums(shells, np.concatenate([pairs, pairs], 1), 0,
                                   "ref" if oeri.ref_available() else "oracle")
        return np.sqrt(np.sqrt(np.maximum(s[:, 0, 1], 0)))
    q = workloads.sample_quartets(shells, min(args.quartets, 1 << 15), seed=1, schwarz_fn=qfn)
    per_step = max(2.0, min(20.0, 120.0 / max(1, args.steps + args.warmup)))
    times = []
    info = None
    for it in range(args.warmup + args.steps):
        info, _, _ = cpu_reference_rate(shells, q, 1, per_step)
        if it >= args.warmup:
            times.append(info["value"])
    v = float(np.mean(times))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "quartets/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "eri_microbench_4096_shells_spd_ip1", "quartets_per_step": "bounded CPU sample",
                       "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": v, "unit": "quartets/s", "cores": info["cores"], "kind": info["kind"],
                             "sample": info["sample"]},
            "e2e": {"value": v, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, ws, rank)
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
        # parity of the measured kernel against the reference build on the CPU subset
        idx = {tuple(r): i for i, r in enumerate(q[:0])}
        gsub = quartet_checksums(ds, torch.from_numpy(sub).to(dev), 1).cpu().numpy()
        l = shells._bas[:, 1][sub]
        nf = np.prod((l + 1) * (l + 2) // 2, axis=1)[:, None].astype(np.float64)
        bound = 2 * np.sqrt(nf * np.abs(ref_vals[..., 1])) + 2e-12 * nf
        parity = float((np.abs(gsub[..., 0] - ref_vals[..., 0]) / bound).max())
        del idx

    tot_q = nq * ws
    value = tot_q / (kernel_ms_max * 1e-3)
    achieved = flops_ip1 / (kernel_ms * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "quartets/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": kernel_ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "eri_microbench_4096_shells_spd_ip1", "nshell": NSHELL, "quartets_per_rank": nq,
                   "lclasses": int(len(classes)), "schwarz": 1e-12,
                   "l2": "256 MiB buffer written between steps, outside the per-step kernel events",
                   "parallelism": "dp%d" % ws if ws > 1 else "single"},
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": "FP64 FMA probe measured in this run (driver peaks file has no FP64 figure)",
                     "flops": "reference-algorithm FP64 op count of the sampled quartets"},
        "int2e_quartets_per_s": tot_q / (int2e_ms * 1e-3),
        "int2e_roofline_frac": flops_int2e / (int2e_ms * 1e-3) / 1e12 / peak,
        "timed_region_ms": region_ms,
        "e2e": {"value": tot_q / (e2e_ms * 1e-3), "unit": "quartets/s", "h2d_bytes_per_step": nq * 16,
                "d2h_bytes_per_step": nq * 3 * 2 * 8},
        "gpu_launches": args.steps,
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "parity_vs_reference_max": parity,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
