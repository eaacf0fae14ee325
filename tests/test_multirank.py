"""The bench's multi-GPU host logic on CPU: two ranks over gloo (127.0.0.1).

With N GPUs the bench runs one independent replica per rank (the simulation
does not shard), times each on its own device and reports the maximum over
ranks, printed by rank 0 alone.  This checks the reduction every rank calls
(bench.max_over_ranks) in a real two-process group, the rank-0-only output,
and that every rank takes the same collective steps."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

WORKER = r"""
import json, os, sys, datetime
sys.path.insert(0, os.environ["ROOT"])
import torch, torch.distributed as dist
import bench
rank = int(os.environ["RANK"])
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
mine = [3.5, 7.25][rank]
got = bench.max_over_ranks(torch, dist, mine, "cpu")
dist.barrier()
if rank == 0:
    print(json.dumps({"max": got, "world": dist.get_world_size()}))
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_two_gloo_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, ROOT=ROOT, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", WORKER], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=240) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e[-2000:]
    assert outs[1][0].strip() == ""  # rank 1 prints nothing
    line = json.loads(outs[0][0].strip().splitlines()[-1])
    assert line == {"max": 7.25, "world": 2}


def test_max_over_ranks_single_process():
    import torch

    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(torch, None, 1.5, "cpu") == 1.5
