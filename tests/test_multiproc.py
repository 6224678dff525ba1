"""The multi-process (replica) path of bench.py on CPU with gloo, world size
2: device times are combined as the maximum over ranks, and the reference
arm run under torchrun prints one JSON line from rank 0 only while the other
rank exits 0 without work."""
import json
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(REPO))
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.barrier(world)
        out[rank] = bench.allreduce_max(1.5 + rank, world)
    finally:
        dist.destroy_process_group()


def test_allreduce_max_gloo():
    import torch.multiprocessing as mp

    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 2.5, 1: 2.5}


def test_reference_arm_rank0_only():
    if not (REPO / "oracle" / "_ref").exists():
        pytest.skip("oracle/_ref not built")
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), str(REPO / "bench.py"),
           "--impl", "reference", "--workload", "plain_16c32", "--gpus", "2", "--steps", "1",
           "--warmup", "0"]
    res = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=REPO, env=env)
    assert res.returncode == 0, res.stderr[-2000:]
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["value"] > 0 and d["unit"] == "solves/s"
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["cpu_baseline"]["kind"] == "reference"
