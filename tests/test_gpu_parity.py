"""GPU parity against the FP64 oracle, through the C ABI.

Tolerances: FP64 mode 1e-9 relative (the reference bar is 1e-6); mixed mode
(FP32 per atom, FP64 sums and grid) 2e-5 relative on CV values and bias, 2e-3
relative on the largest force component.  Neighbour counts are compared
exactly.
"""
import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-9, 1e-9), "mixed": (2e-5, 2e-3)}


def _q_system(seed=11, step=0):
    x, L = systems.config1()
    return systems.jitter(x, 0.15, seed, step), L


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_steinh_q_one_step(precision):
    x, L = _q_system()
    args = H.fix_args_q()
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    cv, bias, f, _ = out[0]
    o = O.steinh_q(6, x, L, 3.9, 18)
    g = O.Grid([[0.0, 1.0]], [1000], 0.01, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([o["cv"]])
    V, dV = g.value([o["cv"]])
    fo = -dV[0] * o["grad"]
    tcv, tf = TOL[precision]
    assert H.rel(cv[0], o["cv"]) < tcv
    assert H.rel(bias, V) < tcv
    assert H.rel(f, fo) < tf
    q = m.extract("Q6.stein_q", x.shape[0])
    assert H.rel(q, o["Q"]) < tcv * 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_local_ql_q4_q6_step(precision):
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = systems.jitter(x, 0.05, 3)
    args = H.fix_args_local()
    m, out = H.run_gpu(args, x, L, [(0, x), (10, x)], precision=precision)
    o4 = H.oracle_local(x, L, 4)
    o6 = H.oracle_local(x, L, 6)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    tcv, tf = TOL[precision]
    for k, (step, _) in enumerate([(0, x), (10, x)]):
        g.add_hill(s)
        V, dV = g.value(s)
        fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
        cv, bias, f, _ = out[k]
        assert H.rel(cv, s) < tcv
        assert H.rel(bias, V) < tcv
        assert H.rel(f, fo) < tf
    assert m.max_neighbors("Q4") == o4["nnb"].max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["MEAN_SOLID", "NSOLID", "FRAC"])
def test_local_ql_smooth_switches(mode, precision):
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = systems.jitter(x, 0.05, 5)
    # NSOLID counts atoms: its grid spans [0, N] with a hill width of a few atoms
    hi, sigma = (800.0, 8.0) if mode == "NSOLID" else (1.0, 0.01)
    args = H.fix_args_local(sw="FERMI", alpha=-8.0, mode=mode, cvsw=(0.35, 20.0), nbins=100, hi=hi, sigma=sigma)
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    swr = O.make_sw("FERMI", r0=3.9, alpha=-8.0)
    rl = O.sw_invert_for_eps(swr, 1e-6)
    swc = O.make_sw("FERMI", r0=0.35, alpha=20.0)
    o4 = O.steinh_l(4, x, L, rl, swr, 1e-6, swc, mode)
    o6 = O.steinh_l(6, x, L, rl, swr, 1e-6, swc, mode)
    g = O.Grid([[0, hi], [0, hi]], [100, 100], sigma, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    g.add_hill(s)
    V, dV = g.value(s)
    fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
    cv, bias, f, _ = out[0]
    tcv, tf = (1e-9, 1e-8) if precision == "fp64" else TOL["mixed"]
    assert H.rel(cv, s) < tcv
    assert H.rel(f, fo) < tf


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_thin_periodic_box(precision):
    """Two cells along z (h >= cutoff, L >= 2 cutoff): the stencil wraps onto
    the same cells, which the general neighbour kernel handles."""
    x = systems.lattice(5, 5, 2, 4.05, systems.FCC_BASIS)
    L = np.array([5 * 4.05, 5 * 4.05, 2 * 4.05])
    x = systems.wrap(systems.jitter(x, 0.08, 9), L)
    args = H.fix_args_local()
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    o4 = H.oracle_local(x, L, 4)
    o6 = H.oracle_local(x, L, 6)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    g.add_hill(s)
    V, dV = g.value(s)
    fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
    cv, bias, f, _ = out[0]
    tcv, tf = TOL[precision]
    assert H.rel(cv, s) < tcv
    assert H.rel(f, fo) < tf
    assert m.max_neighbors("Q4") == o4["nnb"].max()


def _dense_cluster_system():
    """A compact FCC cluster (a = 3.0 A: ~42 neighbours within 3.9 A) in a
    sparse gas: the list width estimated from the mean density is far too
    small, so the first step overflows and is repeated with grown lists."""
    rng = np.random.default_rng(17)
    L = np.array([60.0, 60.0, 60.0])
    cluster = systems.lattice(4, 4, 4, 3.0, systems.FCC_BASIS) + 20.0
    gas = rng.random((200, 3)) * L
    gas = gas[np.min(np.linalg.norm(gas[:, None, :] - cluster[None, :, :], axis=2), axis=1) > 3.0]
    return np.ascontiguousarray(systems.wrap(np.concatenate([cluster, gas]), L)), L


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_neighbour_overflow_is_grown_and_repeated(precision):
    x, L = _dense_cluster_system()
    args = H.fix_args_local()
    m, out = H.run_gpu(args, x, L, [(0, x), (1, x)], precision=precision)
    o4, o6 = H.oracle_local(x, L, 4), H.oracle_local(x, L, 6)
    assert m.max_neighbors("Q4") == o4["nnb"].max() > 30
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    g.add_hill(s)
    V, dV = g.value(s)
    tcv, tf = TOL[precision]
    for cv, bias, f, _ in out:
        assert H.rel(cv, s) < tcv
        assert H.rel(bias, V) < tcv
        assert H.rel(f, -(dV[0] * o4["grad"] + dV[1] * o6["grad"])) < tf


def test_neighbour_overflow_on_the_device_path_asks_for_a_repeat():
    import torch

    x, L = _dense_cluster_system()
    m = mtd.Metad(H.fix_args_local(), precision="fp64")
    m.set_box([0, 0, 0], L)
    dx = torch.from_numpy(x).cuda()
    f = torch.zeros_like(dx)
    m.post_force_device(0, x.shape[0], dx.data_ptr(), f.data_ptr(), f.data_ptr())
    with pytest.raises(mtd.MetadError, match="NEIGH_OVERFLOW"):
        m.sync()
    f.zero_()
    m.post_force_device(0, x.shape[0], dx.data_ptr(), f.data_ptr(), f.data_ptr())
    m.sync()
    o4 = H.oracle_local(x, L, 4)
    assert abs(m.cv[0] - o4["cv"]) < 1e-9 * abs(o4["cv"])


def test_device_path_runs_ahead_and_collects_every_step(tmp_path):
    """Twelve device steps enqueued with no host wait between them (more steps
    than output slots in flight), then one mtd_sync: the HILLS file, the last
    step's CVs and bias and every step's forces equal the host path's."""
    import torch

    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 100, s), L)) for s in range(12)]
    args = H.fix_args_local(pace=2)
    ref = mtd.Metad(args, precision="fp64", hills_path=str(tmp_path / "H1"))
    ref.set_box([0, 0, 0], L)
    f_ref = []
    for s, xv in enumerate(xs):
        f = np.zeros_like(xv)
        ref.post_force(s, xv, f)
        f_ref.append(f)
    cv_ref, bias_ref = ref.cv.copy(), ref.compute_scalar()
    ref.close()
    m = mtd.Metad(args, precision="fp64", hills_path=str(tmp_path / "H2"))
    m.set_box([0, 0, 0], L)
    dxs = [torch.from_numpy(xv).cuda() for xv in xs]
    fs = [torch.zeros_like(d) for d in dxs]
    for s in range(12):
        m.post_force_device(s, xs[s].shape[0], dxs[s].data_ptr(), fs[s].data_ptr(), fs[s].data_ptr())
    m.sync()
    assert np.array_equal(m.cv, cv_ref) and m.compute_scalar() == bias_ref
    m.close()
    assert open(tmp_path / "H1").read() == open(tmp_path / "H2").read()
    for s in range(12):
        assert np.array_equal(fs[s].cpu().numpy(), f_ref[s])
