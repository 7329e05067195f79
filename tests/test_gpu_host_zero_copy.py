"""mtd_post_force on pinned host f with one STEINH L unit and no virial: the
force pass writes f over the host link (zero copy; with host-copy mode 3 it
also reads it there), one thread per caller index so each warp touches one
contiguous stretch of f.  The per-atom arithmetic is the sorted-order pass's,
so forces, CVs and bias equal the device-buffer path (mtd_post_force_device)
bit for bit in every mode.  Pageable host f, or the virial asked for, take
the upload / download path with the same forces."""
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
def test_zero_copy_host_forces_equal_device_path(precision, skin):
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
        fh = torch.from_numpy(f_in.copy()).pin_memory()   # pinned: the zero-copy path
        host.post_force(s, x, fh.numpy())
        dx = torch.from_numpy(x).cuda()
        df_in = torch.from_numpy(f_in).cuda()
        df = torch.empty_like(df_in)
        dev.post_force_device(s, x.shape[0], dx.data_ptr(), df_in.data_ptr(), df.data_ptr())
        dev.sync()
        assert np.array_equal(fh.numpy(), df.cpu().numpy())
        assert np.array_equal(host.cv, dev.cv) and host.compute_scalar() == dev.compute_scalar()
    host.close()
    dev.close()
    # the same first step through every host-copy mode, pageable f and the
    # virial (upload / download path): the same forces
    outs = []
    f0 = np.random.default_rng(7).normal(size=xs[0].shape)   # f_in not zero: the f read is checked too
    for mode in ("copies", "zc_write", "zc_both", "pageable", "virial"):
        m = mtd.Metad(args, precision=precision)
        m.set_box([0, 0, 0], L)
        m.set_host_copy_mode({"copies": 1, "zc_write": 2, "zc_both": 3}.get(mode, 0))
        f = torch.from_numpy(f0.copy())
        f = f.pin_memory() if mode in ("copies", "zc_write", "zc_both") else f
        vir = m.post_force(0, xs[0], f.numpy(), virial=(mode == "virial"))
        outs.append(f.numpy().copy())
        if mode == "virial":
            assert np.all(np.isfinite(vir))
        m.close()
    assert all(np.array_equal(outs[0], o) for o in outs[1:])


def test_default_mode_times_the_modes_and_keeps_the_forces():
    """Mode 0: the first eligible calls run modes 1-3 in turn (one warm-up
    call, then three timed calls each) and the fastest is kept; every call's
    forces equal the device-buffer path's bit for bit whatever mode ran."""
    import torch

    x0, L = _system()
    args = H.fix_args_local(pace=3) + ["NEIGH_SKIN", 0.6]
    host = mtd.Metad(args, precision="mixed")
    dev = mtd.Metad(args, precision="mixed")
    for m in (host, dev):
        m.set_box([0, 0, 0], L)
    assert host.host_copy_mode_in_use() == 0
    for s in range(13):
        x = np.ascontiguousarray(systems.wrap(systems.jitter(x0, 0.02, 300 + s), L))
        f_in = np.random.default_rng(40 + s).normal(size=x.shape)
        fh = torch.from_numpy(f_in.copy()).pin_memory()
        host.post_force(s, x, fh.numpy())
        dx = torch.from_numpy(x).cuda()
        df_in = torch.from_numpy(f_in).cuda()
        df = torch.empty_like(df_in)
        dev.post_force_device(s, x.shape[0], dx.data_ptr(), df_in.data_ptr(), df.data_ptr())
        dev.sync()
        assert np.array_equal(fh.numpy(), df.cpu().numpy()), s
        if s < 9:
            assert host.host_copy_mode_in_use() == 0
    assert host.host_copy_mode_in_use() in (1, 2, 3)
    host.set_host_copy_mode(0)   # a new trial
    assert host.host_copy_mode_in_use() == 0
    host.set_host_copy_mode(2)
    assert host.host_copy_mode_in_use() == 2
    host.close()
    dev.close()
