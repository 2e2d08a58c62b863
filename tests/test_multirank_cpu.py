"""The N > 1 plumbing of bench.py on the host: gloo, world size 2, 127.0.0.1.

* max-over-ranks reduction of the per-rank device times;
* the reference arm under torchrun: rank 0 alone times the reference's CPU
  kernels and prints one JSON line, the other rank exits 0 without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    torch.distributed.init_process_group("gloo", rank=rank, world_size=2)
    try:
        out[rank] = bench._maxr(10.0 + rank, 2, torch.device("cpu"))
    finally:
        torch.distributed.destroy_process_group()


def test_max_over_ranks_gloo():
    out = mp.Manager().dict()
    mp.spawn(_worker, args=(_free_port(), out), nprocs=2, join=True)
    assert out[0] == out[1] == 11.0


def test_reference_arm_under_torchrun_prints_one_line():
    from oracle import eri as oeri
    if not oeri.ref_available():
        pytest.skip("reference kernels not built (run __graft_entry__.build())")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--gpus", "2",
           "--impl", "reference", "--steps", "1", "--warmup", "0", "--quartets", "512"]
    r = subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] in ("reference", "port")
