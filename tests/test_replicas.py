"""The multi-process path of bench.py on the CPU: two gloo ranks.

The SOAP path has no exchange step, so `bench.py --gpus N` runs N independent
replicas; the only collectives are the barrier around the timed region and the
max over ranks of the step time. Both are checked here with world size 2, as
is the reference arm, where rank 0 alone runs and prints and the other rank
exits without work.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

HELPERS = r"""
import json, os, sys
sys.path.insert(0, sys.argv[1])
import bench
rank, world, local = bench.dist_setup(2)
bench.barrier(world)
value = bench.allreduce_max(float(10 + rank), world)
bench.barrier(world)
print(json.dumps({"rank": rank, "world": world, "max": value}))
import torch.distributed as dist
dist.destroy_process_group()
"""


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(args, world=2, timeout=300):
    port = free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="", OMP_NUM_THREADS="2")
        procs.append(subprocess.Popen([sys.executable] + args, env=env, cwd=ROOT, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=timeout)
        assert p.returncode == 0, err[-2000:]
        outs.append(out)
    return outs


def test_barrier_and_max_over_ranks():
    outs = run_ranks(["-c", HELPERS, ROOT])
    lines = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    assert sorted(x["rank"] for x in lines) == [0, 1]
    assert all(x["world"] == 2 and x["max"] == 11.0 for x in lines)


@pytest.mark.timeout(600)
def test_reference_arm_prints_on_rank_zero_only():
    outs = run_ranks([os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2", "--steps", "1",
                      "--warmup", "0", "--atoms", "64"])
    printed = [o.strip() for o in outs]
    assert printed[1] == ""
    line = json.loads(printed[0].splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
