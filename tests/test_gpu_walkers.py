"""Multiple walkers sharing one grid (mtd_walkers_*), through the C ABI, against
the FP64 oracle: every walker's CVs from its own atoms, WT heights from the
grid as it stood at the start of the step, hills deposited in walker order,
V and dV/ds on the updated grid, forces.  FP64 mode: 1e-9 relative on CVs and
bias, 1e-8 on forces.  The CUDA-graph path must reproduce the plain launches
bit for bit."""
import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu


def _walker_systems():
    out = []
    for k, (nxy, nzf, nzb, nliq) in enumerate([(5, 2, 3, 120), (6, 3, 4, 300), (5, 3, 2, 200)]):
        x, L = systems.small_slab(seed=20 + k, nxy=nxy, nz_fcc=nzf, nz_bcc=nzb, n_liq=nliq)
        out.append((np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 30 + k), L)), L))
    return out


def _run(args, syss, steps, graph, hills_path=""):
    import torch

    W = mtd.Walkers(len(syss), args, precision="fp64", hills_path=hills_path)
    for k, (x, L) in enumerate(syss):
        W.set_box(k, [0, 0, 0], L)
    W.init()
    W.enable_graph(graph)
    dx = [torch.from_numpy(x).cuda() for x, _ in syss]
    df = [torch.zeros_like(v) for v in dx]
    out = []
    for step in steps:
        for v in df:
            v.zero_()
        W.step_device(step, [x.shape[0] for x, _ in syss], [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
        W.sync()
        out.append([(W.cv(k, 2), W.bias(k), df[k].cpu().numpy()) for k in range(len(syss))])
    grid = W.grid(200 * 200)
    W.close()
    return out, grid


def test_walkers_match_oracle_synchronous_deposit():
    syss = _walker_systems()
    steps = [0, 1, 2, 3]
    out, grid = _run(H.fix_args_local(pace=2), syss, steps, graph=False)
    ref = [(H.oracle_local(x, L, 4), H.oracle_local(x, L, 6)) for x, L in syss]
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [[o4["cv"], o6["cv"]] for o4, o6 in ref]
    for i, step in enumerate(steps):
        if step % 2 == 0:
            heights = [0.005 * np.exp(-g.value(sw)[0] / (300.0 * 8.617343e-5 * 8.0)) for sw in s]
            for sw, w in zip(s, heights):
                g.deposit(sw, w)
        for k, (o4, o6) in enumerate(ref):
            V, dV = g.value(s[k])
            cv, bias, f = out[i][k]
            assert H.rel(cv, s[k]) < 1e-9
            assert H.rel(bias, V) < 1e-9
            assert H.rel(f, -(dV[0] * o4["grad"] + dV[1] * o6["grad"])) < 1e-8
    assert H.rel(grid, g.grid) < 1e-12


def test_walkers_graph_replay_is_bitwise_identical():
    syss = _walker_systems()
    steps = list(range(6))
    plain, g1 = _run(H.fix_args_local(pace=2), syss, steps, graph=False)
    graph, g2 = _run(H.fix_args_local(pace=2), syss, steps, graph=True)
    for a, b in zip(plain, graph):
        for (cv1, b1, f1), (cv2, b2, f2) in zip(a, b):
            assert np.array_equal(cv1, cv2) and b1 == b2 and np.array_equal(f1, f2)
    assert np.array_equal(g1, g2)


def test_walkers_hills_file_in_walker_order(tmp_path):
    syss = _walker_systems()
    path = str(tmp_path / "HILLS")
    out, _ = _run(H.fix_args_local(pace=2), syss, range(4), graph=False, hills_path=path)
    rows = [l.split() for l in open(path) if not l.startswith("#")]
    assert len(rows) == 2 * len(syss)
    for r, (step, k) in zip(rows, [(0, 0), (0, 1), (0, 2), (2, 0), (2, 1), (2, 2)]):
        assert int(r[0]) == step
        cv = out[step][k][0]
        assert abs(float(r[1]) - cv[0]) < 1e-12 and abs(float(r[2]) - cv[1]) < 1e-12


def test_walkers_overflow_leaves_no_hill_and_no_force():
    """One walker's neighbour lists overflow on the first step: the group step
    reports it, deposits nothing and leaves every force untouched; the
    repeated step then matches the oracle."""
    import torch
    import test_gpu_parity as P

    syss = [P._dense_cluster_system(), _walker_systems()[0]]
    W = mtd.Walkers(2, H.fix_args_local(pace=2), precision="fp64")
    for k, (x, L) in enumerate(syss):
        W.set_box(k, [0, 0, 0], L)
    dx = [torch.from_numpy(x).cuda() for x, _ in syss]
    df = [torch.zeros_like(v) for v in dx]
    ns = [x.shape[0] for x, _ in syss]
    W.step_device(0, ns, [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
    with pytest.raises(mtd.MetadError, match="NEIGH_OVERFLOW"):
        W.sync()
    assert all(float(v.abs().max()) == 0.0 for v in df)
    assert float(np.abs(W.grid(200 * 200)).max()) == 0.0
    W.step_device(0, ns, [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
    W.sync()
    ref = [(H.oracle_local(x, L, 4), H.oracle_local(x, L, 6)) for x, L in syss]
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [[o4["cv"], o6["cv"]] for o4, o6 in ref]
    heights = [0.005 * np.exp(-g.value(sw)[0] / (300.0 * 8.617343e-5 * 8.0)) for sw in s]
    for sw, w in zip(s, heights):
        g.deposit(sw, w)
    for k, (o4, o6) in enumerate(ref):
        V, dV = g.value(s[k])
        assert H.rel(W.cv(k, 2), s[k]) < 1e-9
        assert H.rel(W.bias(k), V) < 1e-9
        assert H.rel(df[k].cpu().numpy(), -(dV[0] * o4["grad"] + dV[1] * o6["grad"])) < 1e-8
    W.close()


def _run_ranks(args, syss, steps, nranks):
    """The same walkers split over nranks thread ranks (equal shares), hills
    exchanged by a host allgather."""
    import threading

    import domain
    import torch

    per = len(syss) // nranks
    red = domain.LocalAllgather(nranks, timeout=120)
    objs = []
    for r in range(nranks):
        W = mtd.Walkers(per, args, precision="fp64")
        W.set_ranks(r, nranks, red.for_rank(r))
        for k in range(per):
            W.set_box(k, [0, 0, 0], syss[r * per + k][1])
        objs.append(W)
    out = [[None] * len(steps) for _ in range(nranks)]
    errs = []

    def run(r):
        try:
            W = objs[r]
            mine = syss[r * per:(r + 1) * per]
            dx = [torch.from_numpy(x).cuda() for x, _ in mine]
            df = [torch.zeros_like(v) for v in dx]
            for i, step in enumerate(steps):
                for v in df:
                    v.zero_()
                W.step_device(step, [x.shape[0] for x, _ in mine], [v.data_ptr() for v in dx],
                              [v.data_ptr() for v in df])
                W.sync()
                out[r][i] = [(W.cv(k, 2), W.bias(k), df[k].cpu().numpy()) for k in range(per)]
        except BaseException as e:
            errs.append(e)
            red.abort()

    th = [threading.Thread(target=run, args=(r,)) for r in range(nranks)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    if errs:
        raise errs[0]
    grids = [W.grid(200 * 200) for W in objs]
    for W in objs:
        W.close()
    return out, grids


def test_walkers_sharded_over_two_ranks_equal_one_group():
    """Four walkers as one group against the same four split 2 + 2 over two
    thread ranks: CVs, bias, forces and the grid bit for bit (each rank
    deposits every rank's hills in global walker order)."""
    base = _walker_systems()
    syss = base + [(np.ascontiguousarray(systems.wrap(systems.jitter(base[0][0], 0.05, 77), base[0][1])),
                    base[0][1])]
    steps = [0, 1, 2, 3]
    args = H.fix_args_local(pace=2)
    one, grid1 = _run(args, syss, steps, graph=False)
    two, grids = _run_ranks(args, syss, steps, 2)
    for i in range(len(steps)):
        for r in range(2):
            for k in range(2):
                cv, b, f = two[r][i][k]
                cv1, b1, f1 = one[i][2 * r + k]
                assert np.array_equal(cv, cv1) and b == b1 and np.array_equal(f, f1)
    assert np.array_equal(grids[0], grids[1]) and np.array_equal(grids[0], grid1)


def test_walkers_sharded_device_allgather_one_rank_nccl():
    """The device-side gather (torch.distributed NCCL all_gather on the
    walkers' stream, world size 1) against the unsharded group, bit for bit."""
    import socket

    import domain
    import torch
    import torch.distributed as dist

    syss = _walker_systems()
    steps = [0, 1, 2]
    args = H.fix_args_local(pace=2)
    one, grid1 = _run(args, syss, steps, graph=False)
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        W = mtd.Walkers(len(syss), args, precision="fp64")
        W.set_ranks_device(0, 1, domain.TorchDeviceAllgather(1))
        for k, (x, L) in enumerate(syss):
            W.set_box(k, [0, 0, 0], L)
        dx = [torch.from_numpy(x).cuda() for x, _ in syss]
        df = [torch.zeros_like(v) for v in dx]
        for i, step in enumerate(steps):
            for v in df:
                v.zero_()
            W.step_device(step, [x.shape[0] for x, _ in syss], [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
            W.sync()
            for k in range(len(syss)):
                cv1, b1, f1 = one[i][k]
                assert np.array_equal(W.cv(k, 2), cv1) and W.bias(k) == b1
                assert np.array_equal(df[k].cpu().numpy(), f1)
        assert np.array_equal(W.grid(200 * 200), grid1)
        W.close()
    finally:
        dist.destroy_process_group()


def test_walkers_with_skin_lists_graph_equals_plain():
    """Skin lists in every walker, the per-walker kernels captured into the
    group's CUDA graph (the list rebuild is then the separate gated kernels)
    against plain launches (the one-launch rebuild): identical steps."""
    syss = _walker_systems()
    args = H.fix_args_local(pace=2) + ["NEIGH_SKIN", 0.6, "NEIGH_EVERY", 3]
    steps = list(range(7))
    plain, g1 = _run(args, syss, steps, graph=False)
    graph, g2 = _run(args, syss, steps, graph=True)
    for a, b in zip(plain, graph):
        for (cv1, b1, f1), (cv2, b2, f2) in zip(a, b):
            assert np.array_equal(cv1, cv2) and b1 == b2 and np.array_equal(f1, f2)
    assert np.array_equal(g1, g2)
