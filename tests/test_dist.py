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


def _tile_rank_main(rank, world, port, out):
    """One rank of the tiled-slab decomposition that `bench.py --gpus N`
    runs: the oracle's STEINH L sums over this rank's owned atoms (ghosts
    are neighbours only), summed over the ranks with gloo."""
    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "metad-toy_b200")]
    import bench
    import oracle as O
    import systems
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        x0, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
        cut = 2 * 3.9 + 1.0
        xs, nown, (lo, hi, per) = bench.tile_rank_positions(x0, L, world, rank, cut, 7, 2)
        st = O.make_sw("STEP", r0=3.9)
        res = []
        for x in xs:
            grp = np.zeros(x.shape[0], np.int32)
            grp[:nown] = 1
            o = O.steinh_l(6, x - np.array(lo), np.array(hi) - np.array(lo), 3.9, st, ingroup=grp,
                           periodic=per, grad=False)
            t = torch.tensor(o["sums"], dtype=torch.float64)
            dist.all_reduce(t)
            res.append(t.numpy().tolist())
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_bench_tiled_decomposition_matches_the_whole_system():
    """Two gloo ranks, each owning one tile of a slab tiled twice along x with
    the ghost shell of STEINH L plus the skin: the summed totals give the
    CV of the undecomposed periodic two-tile system (FP64 oracle, 1e-12)."""
    import numpy as np

    sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "metad-toy_b200")]
    import bench
    import oracle as O
    import systems
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_tile_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    x0, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    Lg = np.array([world * L[0], L[1], L[2]])
    st = O.make_sw("STEP", r0=3.9)
    for c in range(2):
        tiles = [bench.tile_rank_positions(x0, L, world, r, 0.0, 7, 2)[0][c][: x0.shape[0]] + [r * L[0], 0, 0]
                 for r in range(world)]
        og = O.steinh_l(6, np.concatenate(tiles), Lg, 3.9, st, grad=False)
        for r in range(world):
            s = res[r][c]
            assert s[2] == world * x0.shape[0]
            assert abs(s[0] / s[1] - og["cv"]) < 1e-12 * og["cv"]
