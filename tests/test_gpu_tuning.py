"""Autotuner (mtd_autotune, mtd_walkers_autotune): every interchangeable
kernel shape gives bitwise-identical steps, and tuning itself records no step
and deposits nothing."""
import numpy as np
import pytest

import helpers as H
import mtd
import systems

pytestmark = pytest.mark.gpu

SHAPES = [(0, 0, 0), (1, 128, 128), (2, 256, 128), (2, 128, 256)]


def _run(args, x, L, shape, precision, steps=3):
    m = mtd.Metad(args, precision=precision)
    m.set_box([0, 0, 0], L)
    if shape is not None:
        m.set_tuning(*shape)
    out = []
    for step in range(steps):
        f = np.zeros_like(x)
        m.post_force(step, x, f)
        out.append((m.cv.copy(), m.compute_scalar(), f))
    m.close()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_every_shape_gives_identical_steps(precision):
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 31), L))
    args = H.fix_args_local(pace=1)
    ref = _run(args, x, L, None, precision)
    for shape in SHAPES[1:]:
        got = _run(args, x, L, shape, precision)
        for (c1, b1, f1), (c2, b2, f2) in zip(ref, got):
            assert np.array_equal(c1, c2) and b1 == b2 and np.array_equal(f1, f2), shape


def test_shapes_agree_for_capped_lists():
    x, L = systems.config1()
    x = np.ascontiguousarray(systems.jitter(x, 0.15, 5, 0))
    ref = _run(H.fix_args_q(), x, L, None, "fp64")
    for shape in SHAPES[1:]:
        got = _run(H.fix_args_q(), x, L, shape, "fp64")
        for (c1, b1, f1), (c2, b2, f2) in zip(ref, got):
            assert np.array_equal(c1, c2) and b1 == b2 and np.array_equal(f1, f2), shape


def test_autotune_changes_nothing_but_the_shapes(tmp_path):
    import torch

    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 32), L))
    args = H.fix_args_local(pace=1)
    ref = _run(args, x, L, None, "mixed")
    m = mtd.Metad(args, precision="mixed", hills_path=str(tmp_path / "HILLS"))
    m.set_box([0, 0, 0], L)
    dx = torch.from_numpy(x).cuda()
    choice = m.autotune(x.shape[0], dx.data_ptr(), reps=3)
    assert choice[0] in (0, 1, 2) and choice[1] in (128, 256) and choice[2] in (128, 256)
    assert not [l for l in open(tmp_path / "HILLS") if not l.startswith("#")]   # tuning deposited nothing
    for step, (c1, b1, f1) in enumerate(ref):
        f = np.zeros_like(x)
        m.post_force(step, x, f)
        assert np.array_equal(m.cv, c1) and m.compute_scalar() == b1 and np.array_equal(f, f1)
    m.close()


def test_walkers_autotune_keeps_the_steps():
    import torch

    syss = [systems.walker_system(n, 200 + k) for k, n in enumerate([2500, 9000, 4000])]
    ns = [x.shape[0] for x, _ in syss]
    args = ["GAUSSIAN", 0.01, 0.005, 9.0, "PACE", 1, "TEMP", 300.0,
            "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "Q4", "STEINH", "L", 4, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "SYMBOL", "v1", "Q4.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID",
            "CV_dim", 2, "DIM", 1, 0, 1, 100, "v1", "DIM", 2, 0, 1, 100, "v2", "WT", 1]
    results = []
    for tune in (False, True):
        W = mtd.Walkers(len(syss), args, precision="mixed")
        for k, (_, L) in enumerate(syss):
            W.set_box(k, [0, 0, 0], L)
        W.init()
        dx = [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x, _ in syss]
        df = [torch.zeros_like(v) for v in dx]
        if tune:
            picks = W.autotune(ns, [v.data_ptr() for v in dx], reps=3)
            assert len(picks) == 3
        run = []
        for step in range(3):
            for v in df:
                v.zero_()
            W.step_device(step, ns, [v.data_ptr() for v in dx], [v.data_ptr() for v in df])
            W.sync()
            run.append(([W.cv(k, 2).tolist() for k in range(3)], [v.cpu().numpy() for v in df]))
        W.close()
        results.append(run)
    for (cv1, f1), (cv2, f2) in zip(*results):
        assert cv1 == cv2
        assert all(np.array_equal(a, b) for a, b in zip(f1, f2))


def test_sk_tiles_give_identical_steps_and_autotune_picks_one():
    """STRU_FACTOR_K in mixed precision: every k-tile of the value pass (4, 8,
    16) and unroll depth of the force pass (1, 2, 4) gives bitwise-identical
    CVs, bias, forces and virial; mtd_autotune picks one of them."""
    import torch

    x = systems.jitter(systems.fcc(10, 5.26), 0.2, 61)
    L = np.array([10 * 5.26] * 3)
    x = np.ascontiguousarray(systems.wrap(x, L))
    args = ["GAUSSIAN", 0.5, 0.005, 10.0, "PACE", 1,
            "CAL", "NAME", "SK", "STRU_FACTOR_K", "all", "nk", 40, "kmag", systems.KMAG_111, "seed", 5,
            "SYMBOL", "v1", "SK.AVE", "CV_dim", 1, "DIM", 1, 0.0, 100.0, 500, "v1", "WT", 0]

    def run(tiles):
        m = mtd.Metad(args, precision="mixed")
        m.set_box([0, 0, 0], L)
        if tiles is not None:
            m.set_sk_tiles(*tiles)
        out = []
        for step in range(2):
            f = np.zeros_like(x)
            vir = m.post_force(step, x, f, virial=True)
            out.append((m.cv.copy(), m.compute_scalar(), f, np.array(vir)))
        m.close()
        return out

    ref = run(None)
    for tiles in [(4, 1), (16, 4), (8, 1), (4, 4), (16, 2)]:
        got = run(tiles)
        for a, b in zip(ref, got):
            assert all(np.array_equal(u, v) for u, v in zip(a, b)), tiles
    m = mtd.Metad(args, precision="mixed")
    m.set_box([0, 0, 0], L)
    dx = torch.from_numpy(x).cuda()
    m.autotune(x.shape[0], dx.data_ptr(), reps=2)
    qv, qf = m.sk_tiles()
    assert qv in (4, 8, 16) and qf in (1, 2, 4)
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_skin_q_filter_split_and_merged_are_identical(precision):
    """With skin lists the q pass filters the candidates merged with the sum
    (split 0) or in a loop of its own before it (split 1): the same steps bit
    for bit, for both block shapes."""
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.04, 70 + s), L)) for s in range(4)]
    args = H.fix_args_local(pace=2) + ["NEIGH_SKIN", 0.6]

    def run(shape):
        m = mtd.Metad(args, precision=precision)
        m.set_box([0, 0, 0], L)
        m.set_tuning_all(*shape)
        out = []
        for step, xv in enumerate(xs):
            f = np.zeros_like(xv)
            m.post_force(step, xv, f)
            out.append((m.cv.copy(), m.compute_scalar(), f))
        m.close()
        return out

    ref = run((0, 256, 256, 0, 8, 2))
    for shape in [(0, 256, 256, 1, 8, 2), (1, 128, 128, 1, 8, 2), (0, 128, 256, 0, 8, 2)]:
        for (c1, b1, f1), (c2, b2, f2) in zip(ref, run(shape)):
            assert np.array_equal(c1, c2) and b1 == b2 and np.array_equal(f1, f2), shape
