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


GRAD_CHILD = r"""
import json, os, sys
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "optical-flow-filter_b200"))
import torch
import torch.distributed as dist
from flowfilter_b200 import diff
dist.init_process_group("gloo")
rank = dist.get_rank()
g = torch.full((2,), float(rank + 1), dtype=torch.float64)          # a gamma gradient
w = torch.arange(10, dtype=torch.float64).reshape(2, 5) * (rank + 1)   # a weights gradient
loss = torch.tensor([4.0 * rank])
n = diff.average_over_ranks([g, w, loss])
dist.destroy_process_group()
print(json.dumps({"rank": rank, "n": n, "g": g.tolist(), "w": w.tolist(), "loss": loss.tolist()}))
"""


def test_data_parallel_fit_averages_gradients_over_ranks():
    """DiffPyramidalFlowFilter.fit's all-reduce (diff.average_over_ranks), world size 2 over
    gloo: every rank ends with the mean of the ranks' gradients and losses, so all take the
    same Adam step."""
    port = free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", GRAD_CHILD.replace("ROOT", repr(ROOT))], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(json.loads(out.strip().splitlines()[-1]))
    for o in outs:
        assert o["n"] == 2
        assert o["g"] == [1.5, 1.5]
        assert o["w"] == [[1.5 * k for k in range(5)], [1.5 * k for k in range(5, 10)]]
        assert o["loss"] == [2.0]


def test_average_over_ranks_is_a_no_op_without_a_process_group():
    import torch

    from flowfilter_b200 import diff

    t = torch.tensor([1.0, 2.0])
    assert diff.average_over_ranks([t]) == 1 and t.tolist() == [1.0, 2.0]


def test_batch_streams_split_over_ranks_by_compulsory_bytes():
    """BatchFlowFilter.shard: every stream of the benchmark's 64-stream mix on exactly one
    rank, the ranks' compulsory bytes within one largest stream of each other."""
    import bench
    from flowfilter_b200 import BatchFlowFilter

    # the per-frame compulsory bytes of the 2048x1088 three-level workload
    assert BatchFlowFilter.streamBytes(1088, 2048, 3) == 122_552_320
    shapes = [(s["H"], s["W"], s["levels"]) for s in bench.batched_streams()]
    biggest = max(BatchFlowFilter.streamBytes(*s) for s in shapes)
    for ranks in (1, 2, 4, 8):
        parts = BatchFlowFilter.shard(shapes, ranks)
        assert len(parts) == ranks and sorted(i for p in parts for i in p) == list(range(len(shapes)))
        loads = [sum(BatchFlowFilter.streamBytes(*shapes[i]) for i in p) for p in parts]
        assert max(loads) - min(loads) <= biggest
