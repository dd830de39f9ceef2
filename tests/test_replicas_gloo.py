"""The multi-GPU path of bench.py is independent replicas (no data-path
collective): each rank times its own replica, the job's time is the max over
ranks and the job's rate counts every replica's cells.  This runs that
aggregation with two gloo ranks on the CPU, and checks that the reference
arm does its work on rank 0 only."""
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


def _rank(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local_ms = 10.0 + 5.0 * rank            # rank 1 is the slow replica
    ms = bench.max_over_ranks(local_ms, dist, "cpu")
    q.put((rank, ms, bench.job_rate(world, 1000, 4, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for rank, ms, rate in out:
        assert ms == 15.0, (rank, ms)
        assert rate == pytest.approx(2 * 1000 * 4 / 15e-3 / 1e9)


def test_reference_arm_runs_on_rank_zero_only(tmp_path):
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_job_rate_single_replica_matches_definition():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.0, None, "cpu") == 3.0
    assert bench.job_rate(1, 512 ** 3, 200, 500.0) == pytest.approx(512 ** 3 * 200 / 0.5 / 1e9)
    line = {"value": bench.job_rate(1, 10, 1, 1.0)}
    json.dumps(line)
