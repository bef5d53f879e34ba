"""The host side of `bench.py --gpus N` on CPU: N = 2 `gloo` ranks each time an
independent chain ("replicas only", no data-path collective); the reported
time is the slowest rank's and the value is the whole job's throughput.  The
reference arm runs on rank 0 only."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms_rank = [12.5, 17.25][rank]  # each rank's own timed region
        ms = bench.max_over_ranks(ms_rank, dist, "cpu")
        value = bench.job_throughput(world, 10, ms)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"ms": ms, "value": value}, f)
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    got = [json.load(open(tmp_path / f"rank{r}.json")) for r in range(2)]
    for g in got:
        assert g["ms"] == 17.25  # the slowest rank, seen by every rank
        assert abs(g["value"] - 2 * 10 / 0.01725) < 1e-9


def test_single_rank_helpers():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5
    assert abs(bench.job_throughput(1, 5, 250.0) - 20.0) < 1e-12


def test_reference_arm_other_ranks_exit_without_work():
    """Under torchrun every rank but 0 of the reference arm exits 0 without output."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
