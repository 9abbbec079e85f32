"""Multi-GPU is replicas only: each rank steps its own structure and
bench.py reports the whole-job rate over the slowest rank's device time.
These tests run that host logic on two `gloo` ranks on the CPU: the
max-over-ranks reduction every rank takes at the same point, the whole-job
rate, and the reference arm's ranks other than 0 leaving without work."""
import os
import socket
import subprocess
import sys

import pytest

from tests.conftest import ROOT

WORLD = 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_dir):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank device times of 20 replica steps (rank 1 is the slow one)
        local_ms = [400.0, 520.0][rank]
        slowest = bench.max_over_ranks(local_ms, dist, "cpu")
        rate = bench.replica_rate(20, WORLD, slowest / 1000.0)
        # a second reduction at the same point on every rank (the e2e leg)
        e2e_s = bench.max_over_ranks([1.5, 1.25][rank], dist, "cpu")
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{slowest} {rate} {e2e_s}\n")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_time_and_the_whole_job_rate(tmp_path):
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(_free_port(), str(tmp_path)), nprocs=WORLD, start_method="spawn")
    for rank in range(WORLD):
        slowest, rate, e2e_s = map(float, (tmp_path / f"rank{rank}.txt").read_text().split())
        assert slowest == 520.0
        assert rate == pytest.approx(WORLD * 20 / 0.52)
        assert e2e_s == 1.5


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.25, None, "cpu") == 3.25
    assert bench.replica_rate(10, 1, 0.5) == 20.0


def test_reference_arm_ranks_other_than_zero_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
