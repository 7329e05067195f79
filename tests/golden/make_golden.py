"""Generates the golden fixtures in this directory from the reference checkout.

Run in a container that has the reference checkout, after
`make -C oracle ref REF_DIR=<checkout>`:

    python tests/golden/make_golden.py <checkout>      (or REF_DIR=<checkout> in the environment)

Outputs (committed):
  ylm_reference.npz          Y_lm (l = 3, 4, 6) and dY_lm/dd (l = 4, 6) at 256
                             seeded bond vectors, computed by the reference's
                             own CV_Steinhardt_math.h compiled for the host
                             (oracle/_ref/libmtdref.so).
  q_grad_reference_faithful.npz
                             the reference STEINH Q AVE gradient (truncated
                             per-pair terms) on a jittered 108-atom FCC, for
                             documenting the deviation of the exact gradient.
  HILLS_1d_reference_fixture the reference's test/test_cvset/HILLS data file
                             (238 hills), a HILLS-format and replay fixture.
"""
import ctypes as C
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "metad-toy_b200")]

import oracle as O  # noqa: E402
import systems  # noqa: E402


def main(ref_dir=None):
    ref_dir = ref_dir or os.environ.get("REF_DIR")
    if not ref_dir:
        raise SystemExit("usage: make_golden.py <reference checkout>  (or set REF_DIR)")
    R = O.ref_lib()
    if R is None:
        raise SystemExit("build oracle/_ref first: make -C oracle ref")
    rng = np.random.default_rng(20241203)
    d = rng.normal(size=(256, 3)) * rng.uniform(2.0, 4.5, size=(256, 1))
    out = {"d": d}
    dp = C.POINTER(C.c_double)
    for l in (3, 4, 6):
        y = np.zeros((256, 2 * (l + 1)))
        for i in range(256):
            R.ref_ylm(l, *d[i], y[i].ctypes.data_as(dp))
        out["ylm%d" % l] = y
    for l in (4, 6):
        g = np.zeros((256, 6 * (l + 1)))
        for i in range(256):
            R.ref_dylm(l, *d[i], g[i].ctypes.data_as(dp))
        out["dylm%d" % l] = g
    np.savez(os.path.join(HERE, "ylm_reference.npz"), **out)

    # reference-faithful STEINH Q gradient on a jittered 3x3x3 FCC
    x = systems.jitter(systems.fcc(3, 5.26), 0.15, 7)
    L = np.array([3 * 5.26] * 3)
    faithful = {"x": x, "L": L}
    for l in (4, 6):
        o = O.steinh_q(l, x, L, 3.9, 18)
        n, cap = x.shape[0], 18
        disp = np.zeros((n, cap, 3))
        box = O.make_box(L)
        for i in range(n):
            for t in range(o["nkept"][i]):
                dd = np.zeros(3)
                O.lib().orc_minimg(C.byref(box), x[i].ctypes.data_as(dp), x[o["kept"][i, t]].ctypes.data_as(dp),
                                   dd.ctypes.data_as(dp))
                disp[i, t] = dd
        dc = np.zeros((n, 3))
        kept = np.ascontiguousarray(o["kept"], dtype=np.int32)
        nk = np.ascontiguousarray(o["nkept"], dtype=np.int32)
        q = np.ascontiguousarray(o["qlm"])
        Q = np.ascontiguousarray(o["Q"])
        grp = np.ones(n, np.int32)
        ip = C.POINTER(C.c_int)
        R.ref_q_grad_faithful(l, n, cap, kept.ctypes.data_as(ip), nk.ctypes.data_as(ip),
                              disp.ctypes.data_as(dp), q.ctypes.data_as(dp), Q.ctypes.data_as(dp),
                              grp.ctypes.data_as(ip), n, dc.ctypes.data_as(dp))
        faithful["grad_ref%d" % l] = dc
        faithful["grad_exact%d" % l] = o["grad"]
    np.savez(os.path.join(HERE, "q_grad_reference_faithful.npz"), **faithful)

    shutil.copyfile(os.path.join(ref_dir, "test", "test_cvset", "HILLS"),
                    os.path.join(HERE, "HILLS_1d_reference_fixture"))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(*sys.argv[1:])
