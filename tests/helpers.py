"""Helpers shared by the parity tests: run one step through the C ABI and the
same step through the FP64 oracle."""
import numpy as np

import mtd
import oracle as O


def fix_args_q(l=6, rc=3.9, cap=18, sigma=0.01, h=0.005, biasf=10.0, pace=10, wt=0, nbins=1000, lo=0.0, hi=1.0):
    return ["GAUSSIAN", sigma, h, biasf, "PACE", pace,
            "CAL", "NAME", "Q%d" % l, "STEINH", "Q", l, "all", "cutoff_r", rc, "cutoff_Natoms", cap,
            "SYMBOL", "v1", "Q%d.AVE" % l, "CV_dim", 1, "DIM", 1, lo, hi, nbins, "v1", "WT", wt]


def fix_args_local(rc=3.9, sw="STEP", sigma=0.01, h=0.005, biasf=9.0, temp=300.0, pace=10, wt=1, nbins=200,
                   alpha=-8.0, mode="MEAN_SOLID", cvsw=None, lo=0.0, hi=1.0):
    args = ["GAUSSIAN", sigma, h, biasf, "PACE", pace, "TEMP", temp]
    if sw == "STEP":
        args += ["CAL", "NAME", "SWR", "SW_FUNC", "STEP", "r_0", rc]
    else:
        args += ["CAL", "NAME", "SWR", "SW_FUNC", "FERMI", "r_0", rc, "alpha", alpha]
    if cvsw is not None:
        args += ["CAL", "NAME", "SWC", "SW_FUNC", "FERMI", "r_0", cvsw[0], "alpha", cvsw[1]]
    for l in (4, 6):
        args += ["CAL", "NAME", "Q%d" % l, "STEINH", "L", l, "all", "cutoff_r", rc, "cutoff_Natoms", 18,
                 "SW_FUNC_r", "SWR"]
    suffix = ".SWC" if cvsw is not None else ""
    args += ["SYMBOL", "v1", "Q4.%s%s" % (mode, suffix), "SYMBOL", "v2", "Q6.%s%s" % (mode, suffix),
             "CV_dim", 2, "DIM", 1, lo, hi, nbins, "v1", "DIM", 2, lo, hi, nbins, "v2", "WT", wt]
    return args


def run_gpu(args, x, L, steps, precision="fp64", f0=None, virial=False, groups=None, mask=None):
    """Runs `steps` (list of (step, x)) and returns per-step (cv, bias, f, virial)."""
    m = mtd.Metad(args, precision=precision, groups=groups)
    m.set_box([0, 0, 0], L)
    out = []
    for step, xs in steps:
        f = np.zeros_like(xs) if f0 is None else f0.copy()
        v = m.post_force(step, np.ascontiguousarray(xs), f, mask=mask, virial=virial)
        out.append((m.cv.copy(), m.compute_scalar(), f, v))
    return m, out


def oracle_local(x, L, l, rc=3.9, sw=None, mode="MEAN_SOLID", swcv=None, ingroup=None):
    sw = sw or O.make_sw("STEP", r0=rc)
    return O.steinh_l(l, x, L, rc, sw, 1e-6, swcv, mode, ingroup=ingroup)


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))
