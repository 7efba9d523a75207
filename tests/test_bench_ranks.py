"""The multi-rank host logic of bench.py on CPU: two gloo ranks (world size
2, 127.0.0.1 rendezvous) run the same barrier and max-over-ranks reduction
the GPU ranks run over NCCL, the whole-job throughput counts every rank's
replica against the slowest rank's time, and the reference arm leaves
every rank but rank 0 without work."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, port, out_path):
    import datetime
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=2, timeout=datetime.timedelta(seconds=60))
    bench.barrier(2)
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, 2, torch)  # rank 1 is the slower
    bench.barrier(2)
    with open("%s.%d" % (out_path, rank), "w") as f:
        f.write(repr(ms))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time(tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "ms")
    mp.start_processes(_rank_main, args=(_free_port(), out), nprocs=2, start_method="spawn",
                       join=True)
    got = [float(open("%s.%d" % (out, r)).read()) for r in range(2)]
    assert got == [15.0, 15.0]


def test_job_throughput_counts_every_replica():
    import bench
    # 2 ranks x 1,000 particles x 10 steps in 20 ms (the slowest rank)
    assert bench.job_throughput(1000, 2, 10, 20.0) == pytest.approx(1.0e6)
    assert bench.job_throughput(1000, 1, 10, 20.0) == pytest.approx(0.5e6)


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("LOCAL_RANK", "1")
    # rank 1 returns before reading its arguments, a device or the oracle
    assert bench.reference_arm(None) is None
    assert bench.dist_env() == (2, 1, 1)
