"""Learned bias (mtd_nnbias_*): the device network against its NumPy
restatement (oracle/mlp_oracle.py) and the exact hill sum.

Tolerances: forward V within 2e-3 of max|V| and dV/ds within 5e-3 of its
largest component (the device uses SFU exp in SiLU and FP32 tensor-core
accumulation; a BF16 rounding of h1 can flip by one unit); the parameter
gradient within 2e-2 of each block's largest entry; exact hill sum 1e-12
relative plus the skipped far hills (each below h e^-40).  The fitted
network is checked on 65,536 sampled points.
"""
import numpy as np
import pytest

import mlp_oracle as MO
import mtd
import systems

pytestmark = pytest.mark.gpu


def _random_params(seed):
    rng = np.random.default_rng(seed)
    w = np.zeros(MO.NP, dtype=np.float32)
    w[MO.O_W1:MO.O_B1] = rng.normal(0, np.sqrt(2 / 4), MO.H * MO.IN)
    w[MO.O_B1:MO.O_W2] = rng.normal(0, 0.1, MO.H)
    w[MO.O_W2:MO.O_B2] = rng.normal(0, np.sqrt(2 / MO.H), MO.H * MO.H)
    w[MO.O_B2:MO.O_W3] = rng.normal(0, 0.1, MO.H)
    w[MO.O_W3:MO.O_B3] = rng.normal(0, np.sqrt(1 / MO.H), MO.H)
    w[MO.O_B3] = 0.05
    return w


def _box_points(n, seed):
    rng = np.random.default_rng(seed)
    return systems.CV4_LO + (systems.CV4_HI - systems.CV4_LO) * rng.random((n, 4))


def _block_rel(a, b, lo, hi):
    return float(np.abs(a[lo:hi] - b[lo:hi]).max() / max(np.abs(b[lo:hi]).max(), 1e-30))


def test_exact_hill_sum_matches_oracle():
    c, h, s = systems.cv4_hills(n=500, seed=3)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI)
    nb.add_hills(c, h, s)
    p = _box_points(300, 4)
    V, dV = nb.exact(p)
    Vo, dVo = MO.hill_sum(p, c, h, s)
    skipped = len(h) * h.max() * np.exp(-40.0)
    assert np.abs(V - Vo).max() <= 1e-12 * np.abs(Vo).max() + skipped
    assert np.abs(dV - dVo).max() <= 1e-12 * np.abs(dVo).max() + 10 * skipped / s.min()
    nb.close()


@pytest.mark.parametrize("npts", [1, 200, 1000])
def test_forward_and_input_gradient_match_oracle(npts):
    w = _random_params(11)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI)
    nb.set_params(w, 0.7)
    p = _box_points(npts, 5)
    V, dV = nb.eval(p)
    u = MO.normalise(p, systems.CV4_LO, systems.CV4_HI)
    y, gu = MO.input_grad(w, u)
    Vo = 0.7 * y
    dVo = 0.7 * gu[:, :4] * 2.0 / (systems.CV4_HI - systems.CV4_LO)
    assert np.abs(V - Vo).max() <= 2e-3 * max(np.abs(Vo).max(), 1e-3)
    assert np.abs(dV - dVo).max() <= 5e-3 * np.abs(dVo).max()
    nb.close()


def test_parameter_gradient_matches_oracle():
    w = _random_params(12)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI)
    nb.set_params(w, 1.0)
    p = _box_points(640, 6)
    t = np.sin(3 * p[:, 0]) * np.cos(2 * p[:, 1]) + p[:, 2] * p[:, 3]
    g, loss = nb.loss_grad(p, t, 1.0)
    u = MO.normalise(p, systems.CV4_LO, systems.CV4_HI)
    go, lo = MO.loss_grad(w, u, t)
    assert abs(loss - lo) <= 1e-3 * lo
    for a, b in [(MO.O_W1, MO.O_B1), (MO.O_B1, MO.O_W2), (MO.O_W2, MO.O_B2), (MO.O_B2, MO.O_W3),
                 (MO.O_W3, MO.O_B3), (MO.O_B3, MO.NP)]:
        assert _block_rel(g, go, a, b) < 2e-2, (a, b, _block_rel(g, go, a, b))
    nb.close()


def test_point_evaluation_matches_batch():
    import torch

    c, h, s = systems.cv4_hills(n=2000, seed=8)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI)
    nb.add_hills(c, h, s)
    nb.set_params(_random_params(13), 0.3)
    p = _box_points(1, 9)
    d_s = torch.tensor(p[0], dtype=torch.float64, device="cuda")
    d_v = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_g = torch.zeros(4, dtype=torch.float64, device="cuda")
    nb.point_device(d_s.data_ptr(), d_v.data_ptr(), d_g.data_ptr(), use_nn=1)
    torch.cuda.synchronize()
    V, dV = nb.eval(p)
    assert abs(d_v.item() - V[0]) <= 2e-3 * max(abs(V[0]), 1e-3)
    assert np.abs(d_g.cpu().numpy() - dV[0]).max() <= 5e-3 * np.abs(dV[0]).max()
    nb.point_device(d_s.data_ptr(), d_v.data_ptr(), d_g.data_ptr(), use_nn=0)
    torch.cuda.synchronize()
    Ve, dVe = MO.hill_sum(p, c, h, s)
    skipped = len(h) * h.max() * np.exp(-40.0)   # hills beyond sqrt(80) sigma are skipped
    assert abs(d_v.item() - Ve[0]) <= 1e-12 * abs(Ve[0]) + skipped
    assert np.abs(d_g.cpu().numpy() - dVe[0]).max() <= 1e-12 * np.abs(dVe[0]).max() + 10 * skipped / s.min()
    nb.close()


def test_fit_on_hill_sum_and_fallback():
    """20,000 hills (sigma 0.02, h 0.005 eV) along a seeded 4D CV trajectory:
    the fitted network is checked on 65,536 sampled points.  Measured on B200:
    RMS error ~0.017 eV and max ~0.10 eV on a 0.56 eV landscape after 20,000
    Adam steps -- above the 1e-3 eV tolerance, so `usable` stays false and the
    exact FP64 sum stays in charge; a loose tolerance hands over to the network."""
    c, h, s = systems.cv4_hills(n=20000, seed=5)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI, seed=3)
    nb.add_hills(c, h, s)
    loss0 = nb.fit(ntrain=65536, iters=1, batch=4096, lr=3e-3, seed=1)
    loss = nb.fit(ntrain=262144, iters=20000, batch=8192, lr=3e-3, seed=2)
    assert loss < 0.5 * loss0
    mx, rms = nb.validate(npts=65536, seed=7, tol=1e-3)
    vmax = nb.vscale
    print("nnbias fit: vmax %.4g eV, max err %.3g eV, rms %.3g eV" % (vmax, mx, rms))
    assert rms < 0.05 * vmax
    assert nb.usable == (mx <= 1e-3)
    nb.validate(npts=65536, seed=7, tol=2.0 * mx)
    assert nb.usable
    nb.validate(npts=4096, seed=8, tol=0.0)
    assert not nb.usable
    nb.close()


def test_device_batch_equals_host_batch():
    """mtd_nnbias_eval_device on device-resident points: the exact path equals
    mtd_nnbias_exact bit for bit, the network path equals mtd_nnbias_eval up
    to the input normalisation's last-bit rounding (1e-5 of max|V|)."""
    import torch

    c, h, s = systems.cv4_hills(n=500, seed=3)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI)
    nb.set_params(_random_params(13), 0.7)
    nb.add_hills(c, h, s)
    p = _box_points(1000, 6)
    d_p = torch.from_numpy(np.ascontiguousarray(p)).cuda()
    for use_nn, ref in [(0, nb.exact(p)), (1, nb.eval(p))]:
        v = torch.zeros(len(p), dtype=torch.float64, device="cuda")
        g = torch.zeros((len(p), 4), dtype=torch.float64, device="cuda")
        nb.eval_device(len(p), d_p.data_ptr(), v.data_ptr(), g.data_ptr(), use_nn=use_nn)
        torch.cuda.synchronize()
        V, dV = v.cpu().numpy(), g.cpu().numpy()
        if use_nn == 0:
            assert np.array_equal(V, ref[0]) and np.array_equal(dV, ref[1])
        else:
            assert np.abs(V - ref[0]).max() <= 1e-5 * np.abs(ref[0]).max()
            assert np.abs(dV - ref[1]).max() <= 1e-4 * np.abs(ref[1]).max()
    nb.close()


def test_tensor_core_wait_timeout_path():
    """The tile kernel's bounded-wait failure path, taken safely: with stall
    on, every tile waits (64 polls) on a barrier phase that no commit
    completes, after its real tensor-core batch has finished.  Each of the
    three tile modes (values only, values and input gradient, training) then
    returns MTD_ERR_TIMEOUT with no work left in flight (the tile issued no
    further MMA and released its tensor memory); with stall off the next
    calls equal the evaluations made before."""
    import torch

    w = _random_params(14)
    nb = mtd.NNBias(systems.CV4_LO, systems.CV4_HI)
    nb.set_params(w, 0.5)
    p = _box_points(700, 10)
    t = np.sin(p[:, 0])
    d_p = torch.from_numpy(np.ascontiguousarray(p)).cuda()
    d_v = torch.zeros(len(p), dtype=torch.float64, device="cuda")

    def values_only():
        nb.eval_device(len(p), d_p.data_ptr(), d_v.data_ptr(), 0, use_nn=1)
        nb.sync_device()
        return d_v.cpu().numpy().copy()

    ref_v, ref_g, ref_t = values_only(), nb.eval(p), nb.loss_grad(p, t, 1.0)
    nb.set_wait(64, stall=True)
    with pytest.raises(mtd.MetadError, match="TIMEOUT"):
        values_only()
    with pytest.raises(mtd.MetadError, match="TIMEOUT"):
        nb.eval(p)
    with pytest.raises(mtd.MetadError, match="TIMEOUT"):
        nb.loss_grad(p, t, 1.0)
    nb.set_wait(0, stall=False)
    assert np.array_equal(values_only(), ref_v)
    V, dV = nb.eval(p)
    assert np.array_equal(V, ref_g[0]) and np.array_equal(dV, ref_g[1])
    g, loss = nb.loss_grad(p, t, 1.0)
    assert np.array_equal(g, ref_t[0]) and loss == ref_t[1]
    nb.close()
