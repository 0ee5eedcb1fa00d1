"""The multi-rank path of bench.py on CPU: batch members are independent, so ranks run
replicas and only the timings meet (max over ranks through the process group); under
torchrun the reference arm runs on rank 0 alone and prints one line.  gloo, world size 2,
127.0.0.1."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks(torch, dist, 1.5 + 2.0 * rank, torch.device("cpu"))
        out[rank] = got
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        assert dict(out) == {0: 3.5, 1: 3.5}


def test_max_over_ranks_single():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, None, 2.25, torch.device("cpu")) == 2.25


@pytest.mark.timeout(300)
def test_reference_arm_under_torchrun_prints_once():
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=2",
           "--master-addr", "127.0.0.1", "--master-port", str(port), "bench.py",
           "--impl", "reference", "--workload", "getrf_n32", "--steps", "1", "--warmup", "0",
           "--cpu-seconds", "1", "--gpus", "2"]
    r = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=280)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
