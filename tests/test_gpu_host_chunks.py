"""mtd_post_force on host buffers with one STEINH L unit and no virial runs
the force pass in caller-order chunks and copies each chunk of f to the host
while the next one is computed.  The per-atom arithmetic is the same as the
sorted-order force pass, so forces, CVs and bias equal the device-buffer
path (mtd_post_force_device, sorted order, one force launch) bit for bit;
with the virial asked for, the host path takes the one-launch force pass."""
import numpy as np
import pytest

import helpers as H
import mtd
import systems

pytestmark = pytest.mark.gpu


def _system():
    x, L = systems.small_slab(seed=5, nxy=12, nz_fcc=4, nz_bcc=6, n_liq=3000)
    return np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 51), L)), L


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("skin", [False, True])
def test_chunked_host_forces_equal_device_path(precision, skin):
    import torch

    x0, L = _system()
    assert x0.shape[0] >= 4096
    args = H.fix_args_local(pace=2) + (["NEIGH_SKIN", 0.6] if skin else [])
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x0, 0.02, 90 + s), L)) for s in range(4)]
    host = mtd.Metad(args, precision=precision)
    dev = mtd.Metad(args, precision=precision)
    for m in (host, dev):
        m.set_box([0, 0, 0], L)
    for s, x in enumerate(xs):
        f_in = np.random.default_rng(s).normal(size=x.shape)
        fh = f_in.copy()
        host.post_force(s, x, fh)
        dx = torch.from_numpy(x).cuda()
        df_in = torch.from_numpy(f_in).cuda()
        df = torch.empty_like(df_in)
        dev.post_force_device(s, x.shape[0], dx.data_ptr(), df_in.data_ptr(), df.data_ptr())
        dev.sync()
        assert np.array_equal(fh, df.cpu().numpy())
        assert np.array_equal(host.cv, dev.cv) and host.compute_scalar() == dev.compute_scalar()
    # with the virial the one-launch pass runs; the forces are the same
    x = xs[0]
    f1, f2 = np.zeros_like(x), np.zeros_like(x)
    vir = host.post_force(9, x, f1, virial=True)
    host.post_force(10, x, f2)
    assert np.array_equal(f1, f2) and np.all(np.isfinite(vir))
    host.close()
    dev.close()
