"""The multi-rank host logic of bench.py on CPU: two ranks over gloo.

The path has no exchange step (one grid per GPU, the ensemble's instances
independent), so `bench.py --gpus N` runs N replicas; what spans the ranks
is the timing (the max over ranks of the device times), the whole-job rate
built from it, and who prints: rank 0 alone, and in the reference arm rank 0
alone does any work.  These run here as two gloo processes on 127.0.0.1;
the NCCL run on GPUs calls the same functions with CUDA tensors.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

_WORKER = r"""
import datetime, json, os, sys
sys.path.insert(0, sys.argv[1])
import torch.distributed as dist
import bench
rank, world, _ = bench.dist_env()
dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
ms = [12.5, 17.25][rank]                       # each replica's own device time
ms_max = bench.max_over_ranks(ms, dist, device="cpu")
rate = bench.aggregate_rate(world, 1000, 4, ms_max)
print(json.dumps({"rank": rank, "ms_max": ms_max, "rate": rate}), flush=True)
dist.barrier()
dist.destroy_process_group()
"""


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _spawn(code, world, extra_env=None):
    port = _free_port()
    procs = []
    for rank in range(world):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                   MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), **(extra_env or {}))
        procs.append(subprocess.Popen([sys.executable, "-c", code, ROOT], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    outs = []
    for p in procs:
        out, err = p.communicate(timeout=120)
        assert p.returncode == 0, err
        outs.append(out)
    return outs


def test_max_over_ranks_and_rate_two_ranks():
    """Both ranks agree on the slowest replica's time, and the job's rate is
    N replicas' zone-updates over that time."""
    outs = _spawn(_WORKER, 2)
    lines = [json.loads(o.strip().splitlines()[-1]) for o in outs]
    for ln in lines:
        assert ln["ms_max"] == 17.25
        assert ln["rate"] == pytest.approx(2 * 1000 * 4 / 17.25e-3)


def test_reference_arm_other_ranks_do_no_work():
    """Under torchrun the reference arm runs on rank 0 only; rank 1 returns 0
    at once and prints nothing."""
    code = r"""
import sys
sys.path.insert(0, sys.argv[1])
import bench
class A:  # run_reference reads nothing else before it returns on rank 1
    steps = 2; warmup = 3; gpus = 2
sys.exit(bench.run_reference(A(), None))
"""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, "-c", code, ROOT], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.aggregate_rate(1, 2048 * 4096, 20, 334.0) == pytest.approx(2048 * 4096 * 20 / 0.334)
