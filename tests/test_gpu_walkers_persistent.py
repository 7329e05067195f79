"""The multi-walker step as one persistent kernel launch (mtd_walkers_* with
mtd_walkers_enable_persistent), through the C ABI.

Every phase of the step (cell lists, neighbour lists, q_lm, LQ_lm, CVs, the
group's deposit in walker order, coefficients, forces) runs for all walkers
inside one cooperative launch separated by bounded grid barriers.  It runs the
same per-thread bodies and partial-sum blocks as the per-walker kernels, so
CVs, bias, forces, the grid and the HILLS file must equal the per-walker path
bit for bit, in FP64 and in mixed precision, plain and in a CUDA graph.  A
barrier wait that runs out (a block that never arrives, set up by
mtd_walkers_set_wait's stall switch) must end the launch with MTD_ERR_TIMEOUT
and leave the object usable: the repeated step equals the reference.
"""
import numpy as np
import pytest

import helpers as H
import mtd
import systems

pytestmark = pytest.mark.gpu


def _walker_systems(count=3, seed=20):
    shapes = [(5, 2, 3, 120), (6, 3, 4, 300), (5, 3, 2, 200), (6, 2, 2, 150)]
    out = []
    for k in range(count):
        nxy, nzf, nzb, nliq = shapes[k % len(shapes)]
        x, L = systems.small_slab(seed=seed + k, nxy=nxy, nz_fcc=nzf, nz_bcc=nzb, n_liq=nliq)
        out.append((np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, seed + 10 + k), L)), L))
    return out


def _run(args, syss, steps, persistent, precision="fp64", graph=False, hills_path="", moving=False, bins=200 * 200):
    """Steps every walker through `steps`; returns per step the CVs, bias and
    forces of each walker, the grid at the end, whether the last step ran as
    one launch and the launch count of the last step."""
    import torch

    W = mtd.Walkers(len(syss), args, precision=precision, hills_path=hills_path)
    for k, (x, L) in enumerate(syss):
        W.set_box(k, [0, 0, 0], L)
    W.init()
    W.enable_persistent(persistent)
    W.enable_graph(graph)
    dx = [torch.from_numpy(x).cuda() for x, _ in syss]
    df = [torch.zeros_like(v) for v in dx]
    out = []
    for i, step in enumerate(steps):
        if moving:   # new positions in the same buffers (a graph replays the same pointers)
            for k, (x, L) in enumerate(syss):
                dx[k].copy_(torch.from_numpy(np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.03, 500 + 7 * i + k), L))))
        for v in df:
            v.zero_()
        W.step_device(step, [x.shape[0] for x, _ in syss], [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
        W.sync()
        out.append([(W.cv(k, 2), W.bias(k), df[k].cpu().numpy()) for k in range(len(syss))])
    grid = W.grid(bins)
    info = (W.persistent_active, W.launch_count())
    W.close()
    return out, grid, info


def _assert_identical(a, b):
    (oa, ga, _), (ob, gb, _) = a, b
    for sa, sb in zip(oa, ob):
        for (cv1, b1, f1), (cv2, b2, f2) in zip(sa, sb):
            assert np.array_equal(cv1, cv2), (cv1, cv2)
            assert b1 == b2, (b1, b2)
            assert np.array_equal(f1, f2), float(np.abs(f1 - f2).max())
    assert np.array_equal(ga, gb)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sw", ["STEP", "FERMI"])
def test_persistent_step_equals_per_walker_kernels(sw, precision):
    syss = _walker_systems()
    args = H.fix_args_local(sw=sw, pace=2)
    steps = list(range(6))
    ref = _run(args, syss, steps, persistent=False, precision=precision, moving=True)
    got = _run(args, syss, steps, persistent=True, precision=precision, moving=True)
    assert ref[2][0] is False and ref[2][1] > 1
    assert got[2] == (True, 1)
    _assert_identical(ref, got)


def test_persistent_step_single_orders_and_many_walkers():
    """STEINH L 6 alone (one order) over 12 walkers, deposits every step."""
    syss = _walker_systems(count=12, seed=40)
    args = ["GAUSSIAN", 0.02, 0.004, 8.0, "PACE", 1, "TEMP", 300.0,
            "CAL", "NAME", "SWR", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18, "SW_FUNC_r", "SWR",
            "SYMBOL", "v1", "Q6.MEAN_SOLID", "CV_dim", 1, "DIM", 1, 0, 1, 200, "v1", "WT", 1]
    steps = list(range(4))
    ref = _run(args, syss, steps, persistent=False, moving=True, bins=200)
    got = _run(args, syss, steps, persistent=True, moving=True, bins=200)
    assert got[2] == (True, 1)
    assert np.array_equal(ref[1], got[1])
    for sa, sb in zip(ref[0], got[0]):
        for (cv1, b1, f1), (cv2, b2, f2) in zip(sa, sb):
            assert np.array_equal(cv1[:1], cv2[:1]) and b1 == b2 and np.array_equal(f1, f2)


def test_persistent_graph_replay_is_bitwise_identical():
    syss = _walker_systems()
    args = H.fix_args_local(pace=2)
    steps = list(range(6))
    plain = _run(args, syss, steps, persistent=True, moving=True)
    graph = _run(args, syss, steps, persistent=True, graph=True, moving=True)
    assert graph[2] == (True, 1)
    _assert_identical(plain, graph)


def test_persistent_hills_file_equals_per_walker_path(tmp_path):
    syss = _walker_systems()
    args = H.fix_args_local(pace=2)
    p1, p2 = str(tmp_path / "HILLS.ref"), str(tmp_path / "HILLS.one")
    _run(args, syss, range(5), persistent=False, hills_path=p1)
    _run(args, syss, range(5), persistent=True, hills_path=p2)
    a = [l for l in open(p1) if not l.startswith("#")]
    b = [l for l in open(p2) if not l.startswith("#")]
    assert len(a) == 3 * len(syss) and a == b


def test_barrier_timeout_reports_and_recovers():
    """One block never arrives at the first grid barrier: the others give up
    after the wait limit, the launch ends, sync reports MTD_ERR_TIMEOUT, no
    hill is deposited, and the repeated step equals the reference."""
    import torch

    syss = _walker_systems()
    args = H.fix_args_local(pace=2)
    ref = _run(args, syss, [0], persistent=False)
    W = mtd.Walkers(len(syss), args, precision="fp64")
    for k, (x, L) in enumerate(syss):
        W.set_box(k, [0, 0, 0], L)
    W.init()
    dx = [torch.from_numpy(x).cuda() for x, _ in syss]
    df = [torch.zeros_like(v) for v in dx]
    ns = [x.shape[0] for x, _ in syss]
    W.set_wait(limit=2000, stall=True)
    W.step_device(0, ns, [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
    with pytest.raises(mtd.MetadError, match="TIMEOUT"):
        W.sync()
    assert float(np.abs(W.grid(200 * 200)).max()) == 0.0
    W.set_wait(limit=0, stall=False)
    for v in df:
        v.zero_()
    W.step_device(0, ns, [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
    W.sync()
    assert W.persistent_active
    for k in range(len(syss)):
        cv, b, f = ref[0][0][k]
        assert np.array_equal(W.cv(k, 2), cv) and W.bias(k) == b
        assert np.array_equal(df[k].cpu().numpy(), f)
    assert np.array_equal(W.grid(200 * 200), ref[1])
    W.close()


def test_ineligible_decks_take_the_per_walker_kernels():
    """Skin lists, or a box with fewer than three cells along a periodic side,
    run the per-walker kernels (several launches) with the same results."""
    syss = _walker_systems(count=2)
    args = H.fix_args_local(pace=2) + ["NEIGH_SKIN", 0.5]
    out, _, info = _run(args, syss, [0, 1], persistent=True)
    assert info[0] is False and info[1] > 1
    x = systems.lattice(5, 5, 2, 4.05, systems.FCC_BASIS)
    L = np.array([5 * 4.05, 5 * 4.05, 2 * 4.05])
    thin = [(np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 3 + k), L)), L) for k in range(2)]
    a = _run(H.fix_args_local(pace=2), thin, [0, 1], persistent=True)
    b = _run(H.fix_args_local(pace=2), thin, [0, 1], persistent=False)
    assert a[2][0] is False
    _assert_identical(a, b)
