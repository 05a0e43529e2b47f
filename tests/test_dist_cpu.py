"""The N>1 plumbing of bench.py (one process per GPU, max over ranks, replicas) on CPU:
world size 2 over gloo, as bench.py runs it under torchrun with NCCL on GPUs."""

from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

from conftest import ROOT


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


CHILD = r"""
import json, os, sys
sys.path.insert(0, ROOT)
import bench
world, rank, local = bench.dist_setup()
assert world == 2 and rank == int(os.environ["RANK"])
bench.barrier(world)
slowest = bench.max_over_ranks(world, 10.0 + 5.0 * rank)   # rank 1 is the slow one
rate = bench.aggregate_rate(world, 100, slowest)
import torch.distributed as dist
dist.destroy_process_group()
print(json.dumps({"rank": rank, "slowest": slowest, "rate": rate}))
"""


def test_two_ranks_take_the_max_over_ranks():
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), FFB_DIST_BACKEND="gloo", CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", CHILD.replace("ROOT", repr(ROOT))], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["slowest"] == 15.0  # both ranks see the slowest rank's time
        assert abs(o["rate"] - 2 * 100 / 0.015) < 1e-6  # all ranks' units over the slowest time


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "3",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
