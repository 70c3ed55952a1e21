"""The multi-GPU path of bench.py is replicas only: every rank fits its own
data set, the only collectives are the timing barrier and the max over ranks
of the elapsed time, and the reference arm runs on rank 0 alone.  These
checks run that host logic as two gloo ranks on the CPU."""
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
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # each replica its own data; the job time is the slowest rank's
        x, y, h, _ = bench.workload(bench.replica_seed(rank), 1000)
        local_ms = 10.0 + 5.0 * rank
        job_ms = bench.max_over_ranks(local_ms, world, torch.device("cpu"))
        dist.barrier()
        out.put((rank, float(x[0, 0]), local_ms, job_ms))
    finally:
        dist.destroy_process_group()


def test_replicas_and_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] != res[1][1]                  # different data per replica
    assert all(r[3] == max(v[2] for v in res) for r in res)


def test_reference_arm_runs_on_rank_zero_only():
    """Under torchrun a rank other than 0 exits 0 without work or output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "0"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert p.returncode == 0
    assert p.stdout.strip() == ""


def test_batched_problems_split_between_ranks_by_cost():
    """Problem sharding of the batched workload: every problem goes to
    exactly one rank and the ranks' estimated loads are close."""
    sys.path.insert(0, ROOT)
    import bench
    from fastlpr_b200.plan import estimated_cost, partition_by_cost
    probs = bench.batched_workload(count=64)
    costs = [estimated_cost(*p) for p in probs]
    for world in (1, 2, 4):
        parts = partition_by_cost(costs, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= 1.2 * min(loads)
