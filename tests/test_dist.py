"""Multi-rank paths of bench.py on CPU (gloo), no GPU needed.

The bench runs one replica per GPU and reports the slowest rank's time; the
reference arm runs on rank 0 only and the other ranks exit without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _max_worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks(1.5 + rank, dist, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world_2():
    import torch.multiprocessing as mp
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_max_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    assert out[0] == out[1] == 2.5
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0


def test_reference_arm_under_torchrun_prints_one_line():
    """bench.py --impl reference with two ranks: rank 0 alone runs and prints."""
    pytest.importorskip("torch")
    oracle_lib = os.path.join(ROOT, "oracle", "liboracle.so")
    if not os.path.exists(oracle_lib):
        pytest.skip("oracle not built")
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.join(ROOT, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
