"""Host logic of `bench.py --gpus N` on CPU with the gloo backend, two ranks:
the job time is the maximum over ranks, the throughput counts every rank's
replica, and the reference arm runs on rank 0 only."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks([10.0 + rank, 50.0 - 5 * rank], dist, "cpu")
        out[rank] = (ms, bench.replica_throughput(1000, 4, world, ms[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_weak_scaling_throughput():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    for rank in range(world):
        ms, thr = res[rank]
        assert ms == [11.0, 50.0]
        assert thr == pytest.approx(1000 * 4 * world / 0.011)


def test_reference_arm_runs_on_rank_zero_only():
    sys.path.insert(0, ROOT)
    import argparse

    import bench
    args = argparse.Namespace(gpus=2, steps=1, warmup=1)
    assert bench.run_reference(args, rank=1) == 0
