"""The two-call step of the C ABI (mtd_set_positions_f64, then mtd_step),
mtd_get_peratom and mtd_create_from_config against mtd_post_force on the
same inputs: identical forces, CVs, bias, virial and per-atom values."""
import ctypes as C

import numpy as np
import pytest

import helpers as H
import mtd
import systems

pytestmark = pytest.mark.gpu


def _steps(nsteps=4):
    x0, L = systems.small_slab(nxy=5, nz_fcc=2, nz_bcc=3, n_liq=200)
    return [np.ascontiguousarray(systems.wrap(systems.jitter(x0, 0.05, 70, s), L)) for s in range(nsteps)], L


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_call_step_equals_post_force(precision):
    xs, L = _steps()
    args = H.fix_args_local(pace=2)
    a = mtd.Metad(args, precision=precision)
    b = mtd.Metad(args, precision=precision)
    for m in (a, b):
        m.set_box([0, 0, 0], L)
    mask = np.ones(xs[0].shape[0], dtype=np.int32)
    for s, x in enumerate(xs):
        fa = np.full_like(x, 0.25)
        fb = fa.copy()
        va = a.post_force(s, x, fa, mask=mask, virial=True)
        b.set_positions(x, mask=mask, groupbit=1)
        cv, bias, vb = b.step(s, fb, virial=True)
        assert np.array_equal(fa, fb) and np.array_equal(va, vb)
        assert np.array_equal(cv, a.cv) and bias == a.compute_scalar()
    n = xs[0].shape[0]
    assert np.array_equal(b.get_peratom("Q6.stein_q", n), a.extract("Q6.stein_q", n))
    with pytest.raises(mtd.MetadError, match="mtd_set_positions_f64 first"):
        b.step(len(xs), np.zeros_like(xs[0]))
    with pytest.raises(mtd.MetadError, match="groupbit"):
        b.set_positions(xs[0], groupbit=0)
    a.close()
    b.close()


def test_create_from_config():
    xs, L = _steps(2)
    args = [str(t).encode() for t in H.fix_args_local(pace=1)]
    L_ = mtd.lib()
    cfg = mtd.Config()
    cfg.narg = len(args)
    argv = (C.c_char_p * len(args))(*args)
    cfg.arg = argv
    L_.mtd_options_default(C.byref(cfg.opt))
    cfg.opt.hills_path = b""
    h = C.c_void_p()
    assert L_.mtd_create_from_config(C.byref(cfg), C.byref(h)) == mtd.MTD_OK
    lo, hi, pe = (C.c_double * 3)(0, 0, 0), (C.c_double * 3)(*L), (C.c_int * 3)(1, 1, 1)
    assert L_.mtd_set_box(h, lo, hi, pe) == mtd.MTD_OK
    ref = mtd.Metad(H.fix_args_local(pace=1), precision="mixed")
    ref.set_box([0, 0, 0], L)
    for s, x in enumerate(xs):
        f1, f2 = np.zeros_like(x), np.zeros_like(x)
        assert L_.mtd_post_force(h, s, x.shape[0], x.ctypes.data, None, None, f1.ctypes.data, None) == mtd.MTD_OK
        ref.post_force(s, x, f2)
        assert np.array_equal(f1, f2)
    L_.mtd_destroy(h)
    ref.close()
