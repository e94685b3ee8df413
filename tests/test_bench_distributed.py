"""bench.py's multi-process plumbing on CPU (gloo, world size 2): each rank
runs its own replica and the reported time is the max over ranks; only rank 0
prints."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import json, os, sys
sys.path.insert(0, os.environ["REPO"])
import bench
world, rank, local = bench.dist_setup()
assert (world, rank, local) == (2, int(os.environ["RANK"]), int(os.environ["LOCAL_RANK"]))
bench.barrier(world)
m = bench.barrier_max(1.5 + rank, world)   # rank 1 is the slower replica
if rank == 0:
    print(json.dumps({"max": m}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_max_over_replicas():
    port = free_port()
    procs = []
    for r in range(2):
        env = dict(os.environ, REPO=ROOT, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = [p.communicate(timeout=180) for p in procs]
    for p, (o, e) in zip(procs, outs):
        assert p.returncode == 0, e
    assert json.loads(outs[0][0].strip().splitlines()[-1]) == {"max": 2.5}
    assert outs[1][0].strip() == ""
