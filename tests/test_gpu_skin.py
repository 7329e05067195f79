"""Skin neighbour lists (NEIGH_SKIN / NEIGH_EVERY) against the per-step
rebuild, through the C ABI.

The lists kept across steps must give the same neighbour sets as a rebuild at
every step: the cell list and the candidates (cutoff + skin) are rebuilt when
an atom moved more than skin / 2, and filtered to the exact criterion every
step.  Compared on a drifting, wrapped trajectory: every step's CVs and bias
within 1e-12 (FP64) or 2e-6 (mixed) relative, forces within 1e-10 / 5e-4 of
the largest component, the whole grid at the end, and the per-atom lists at
several steps exactly.  The sums may differ in their last bits only because
the neighbours come in another order.
"""
import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-12, 1e-10), "mixed": (2e-6, 5e-4)}


def _trajectory(steps, seed=31, drift=0.004, jit=0.02):
    """A slab whose atoms drift with fixed seeded velocities plus a fresh
    jitter every step, wrapped into the box (atoms cross periodic faces)."""
    x0, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    rng = np.random.default_rng(seed)
    v = rng.normal(0.0, drift, x0.shape)
    out = []
    for s in range(steps):
        x = x0 + s * v + rng.normal(0.0, jit, x0.shape)
        out.append(np.ascontiguousarray(systems.wrap(x, L)))
    return out, L


def _run(args, xs, L, precision):
    m = mtd.Metad(args, precision=precision)
    m.set_box([0, 0, 0], L)
    res = []
    for s, x in enumerate(xs):
        f = np.zeros_like(x)
        m.post_force(s, x, f)
        lists = m.neighbors("Q4", x.shape[0], max_per_atom=64)[1] if s % 25 == 0 else None
        res.append((m.cv.copy(), m.compute_scalar(), f, lists))
    return m, res


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sw", ["STEP", "FERMI"])
def test_skin_lists_equal_per_step_rebuild(sw, precision):
    xs, L = _trajectory(100)
    base = H.fix_args_local(sw=sw, pace=5)
    ref_m, ref = _run(base, xs, L, precision)
    ref_grid = ref_m.grid(200 * 200)
    ref_m.close()
    m, out = _run(base + ["NEIGH_SKIN", 0.6], xs, L, precision)
    rebuilds, active = m.neighbor_stats()
    grid = m.grid(200 * 200)
    m.close()
    assert active
    assert 2 <= rebuilds < 60, rebuilds   # drift triggers rebuilds, most steps reuse the lists
    tcv, tf = TOL[precision]
    for (cv0, b0, f0, l0), (cv1, b1, f1, l1) in zip(ref, out):
        assert H.rel(cv1, cv0) < tcv
        assert abs(b1 - b0) <= tcv * max(abs(b0), 1e-3)
        assert H.rel(f1, f0) < tf
        if l0 is not None:
            assert np.array_equal(l0, l1)
    assert np.max(np.abs(grid - ref_grid)) <= tcv * np.max(np.abs(ref_grid)) * 10


def test_neigh_every_forces_rebuilds_and_order_changes_are_caught():
    """Still atoms: NEIGH_EVERY 5 rebuilds at steps 0, 5, 10, 15 only.  At
    step 18 (three steps after the last rebuild) a permutation of the
    caller's atoms (same n) moves the slots far from their build positions,
    so that step rebuilds; a new atom count rebuilds too.  Results equal the
    per-step path throughout (FP64, 1e-12)."""
    xs, L = _trajectory(1, jit=0.0)
    x = xs[0]
    n = x.shape[0]
    args = H.fix_args_local(pace=5)
    m = mtd.Metad(args + ["NEIGH_SKIN", 0.6, "NEIGH_EVERY", 5], precision="fp64")
    ref = mtd.Metad(args, precision="fp64")
    for c in (m, ref):
        c.set_box([0, 0, 0], L)

    def step(s, xv):
        f1, f2 = np.zeros_like(xv), np.zeros_like(xv)
        m.post_force(s, xv, f1)
        ref.post_force(s, xv, f2)
        assert H.rel(m.cv, ref.cv) < 1e-12 and H.rel(f1, f2) < 1e-10

    for s in range(18):
        step(s, x)
    assert m.neighbor_stats()[0] == 4
    perm = np.random.default_rng(3).permutation(n)
    step(18, np.ascontiguousarray(x[perm]))
    assert m.neighbor_stats()[0] == 5
    step(19, np.ascontiguousarray(x[perm][: n - 7]))
    assert m.neighbor_stats()[0] == 6
    m.close()
    ref.close()


def test_one_atom_jump_triggers_a_rebuild():
    """One atom moved by 0.35 A (more than skin / 2 = 0.3) between two steps:
    the displacement test opens the gate, the lists are rebuilt, and the
    neighbour lists equal the oracle's exactly."""
    xs, L = _trajectory(1, jit=0.0)
    x = xs[0].copy()
    n = x.shape[0]
    m = mtd.Metad(H.fix_args_local(pace=5) + ["NEIGH_SKIN", 0.6], precision="mixed")
    m.set_box([0, 0, 0], L)
    m.post_force(0, x, np.zeros_like(x))
    m.post_force(1, x, np.zeros_like(x))
    assert m.neighbor_stats()[0] == 1
    x[17] += np.array([0.35, 0.0, 0.0])
    x = np.ascontiguousarray(systems.wrap(x, L))
    m.post_force(2, x, np.zeros_like(x))
    assert m.neighbor_stats()[0] == 2
    off, nbr = O.local_lists(x, L, 3.9, O.make_sw("STEP", r0=3.9))
    counts, lists = m.neighbors("Q6", n, max_per_atom=64)
    assert np.array_equal(counts, np.diff(off)) and np.array_equal(lists[lists >= 0], nbr)
    m.close()


def test_device_path_with_skin_lists():
    """Twelve asynchronous device steps with skin lists equal the host path
    with per-step rebuilds (FP64, 1e-12)."""
    import torch

    xs, L = _trajectory(12)
    args = H.fix_args_local(pace=2)
    ref = mtd.Metad(args, precision="fp64")
    ref.set_box([0, 0, 0], L)
    f_ref = []
    for s, x in enumerate(xs):
        f = np.zeros_like(x)
        ref.post_force(s, x, f)
        f_ref.append(f)
    cv_ref = ref.cv.copy()
    ref.close()
    m = mtd.Metad(args + ["NEIGH_SKIN", 0.6], precision="fp64")
    m.set_box([0, 0, 0], L)
    dxs = [torch.from_numpy(x).cuda() for x in xs]
    fs = [torch.zeros_like(d) for d in dxs]
    for s in range(12):
        m.post_force_device(s, xs[s].shape[0], dxs[s].data_ptr(), fs[s].data_ptr(), fs[s].data_ptr())
    m.sync()
    assert H.rel(m.cv, cv_ref) < 1e-12
    for s in range(12):
        assert H.rel(fs[s].cpu().numpy(), f_ref[s]) < 1e-10
    m.close()


def test_candidate_overflow_is_grown_and_repeated():
    """A dense cluster in a sparse gas: the candidate capacity estimated from
    the mean density is far too small, the first step overflows the
    candidates, grows them and repeats; results equal the per-step path."""
    rng = np.random.default_rng(17)
    L = np.array([60.0, 60.0, 60.0])
    cluster = systems.lattice(4, 4, 4, 3.0, systems.FCC_BASIS) + 20.0
    gas = rng.random((200, 3)) * L
    gas = gas[np.min(np.linalg.norm(gas[:, None, :] - cluster[None, :, :], axis=2), axis=1) > 3.0]
    x = np.ascontiguousarray(systems.wrap(np.concatenate([cluster, gas]), L))
    args = H.fix_args_local()
    m, out = H.run_gpu(args + ["NEIGH_SKIN", 0.8], x, L, [(0, x), (1, x)], precision="fp64")
    r, ref = H.run_gpu(args, x, L, [(0, x), (1, x)], precision="fp64")
    for (cv0, b0, f0, _), (cv1, b1, f1, _) in zip(ref, out):
        assert H.rel(cv1, cv0) < 1e-12 and H.rel(f1, f0) < 1e-10
    rebuilds, active = m.neighbor_stats()
    assert active and rebuilds >= 1   # one per attempt of step 0 (the retry rebuilds with grown lists)
    m.close()
    r.close()


def test_thin_box_falls_back_to_per_step_lists():
    """Two cells along z: the skin lists need three cells of cutoff + skin per
    periodic side, so the context rebuilds every step and says so."""
    x = systems.lattice(5, 5, 2, 4.05, systems.FCC_BASIS)
    L = np.array([5 * 4.05, 5 * 4.05, 2 * 4.05])
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.08, 9), L))
    m, out = H.run_gpu(H.fix_args_local() + ["NEIGH_SKIN", 0.6], x, L, [(0, x)], precision="fp64")
    assert m.neighbor_stats() == (0, False)
    o4 = H.oracle_local(x, L, 4)
    assert H.rel(out[0][0][0], o4["cv"]) < 1e-9
    m.close()


def test_rebuild_barrier_timeout_reports_and_recovers():
    """The skin-list rebuild is one cooperative launch with bounded grid
    barriers.  A block that never arrives (mtd_neighbor_set_wait's stall
    switch) makes the others give up after the wait limit: the step returns
    MTD_ERR_TIMEOUT, deposits no hill, applies no bias force, and the next
    step rebuilds from scratch and equals a run without the stall bit for bit
    (NEIGH_EVERY 1: both runs rebuild every step)."""
    xs, L = _trajectory(4)
    args = H.fix_args_local(pace=2) + ["NEIGH_SKIN", 0.6, "NEIGH_EVERY", 1]
    ref = mtd.Metad(args, precision="fp64")
    ref.set_box([0, 0, 0], L)
    f_ref = []
    for s in range(4):
        f = np.zeros_like(xs[s])
        ref.post_force(s, xs[s], f)
        f_ref.append((ref.cv.copy(), ref.compute_scalar(), f))
    grid_ref = ref.grid(200 * 200)
    ref.close()
    m = mtd.Metad(args, precision="fp64")
    m.set_box([0, 0, 0], L)
    for s in range(2):
        m.post_force(s, xs[s], np.zeros_like(xs[s]))
    grid1 = m.grid(200 * 200)
    m.neighbor_set_wait(limit=2000, stall=True)
    f = np.zeros_like(xs[2])
    with pytest.raises(mtd.MetadError, match="TIMEOUT"):
        m.post_force(2, xs[2], f)
    assert float(np.abs(f).max()) == 0.0
    assert np.array_equal(m.grid(200 * 200), grid1)
    m.neighbor_set_wait(limit=0, stall=False)
    for s in (2, 3):
        f = np.zeros_like(xs[s])
        m.post_force(s, xs[s], f)
        cv, b, fr = f_ref[s]
        assert np.array_equal(m.cv, cv) and m.compute_scalar() == b and np.array_equal(f, fr)
    assert np.array_equal(m.grid(200 * 200), grid_ref)
    m.close()
