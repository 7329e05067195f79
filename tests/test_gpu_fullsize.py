"""Parity at the benchmark sizes, through the C ABI, against the FP64 oracle.

* The headline deck: 256,000 atoms of FCC / BCC / hard-core-liquid slabs
  (the positions the benchmark times), STEINH L Q4 + Q6 MEAN_SOLID, STEP at
  3.9 A, 2D 200 x 200 WT grid, PACE 10.  One deposit step and one
  non-deposit step, in mixed precision (the benchmark's) and in FP64.
  Per-atom neighbour counts and lists must equal the oracle's exactly.
  Stated tolerances (relative): CV 1e-6 in mixed mode (the error target of
  the method) and 1e-9 in FP64; bias 1e-6 / 1e-9; per-atom LQ 1e-5 / 1e-9;
  force 5e-4 / 1e-8 of the largest force component.  The measured errors
  are printed.
* Config 1's protocol: 4,000-atom FCC, STEINH Q 6 (cutoff 3.9, cap 18), FP64,
  1,000 steps of seeded positions, WT 0, PACE 10 (100 hills): every step's
  CV and bias, forces every 50 steps and the whole 1,000-bin grid at the end.
"""
import json

import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu

KB = 8.617343e-5
TOL = {"mixed": dict(cv=1e-6, bias=1e-6, lq=1e-5, force=5e-4),
       "fp64": dict(cv=1e-9, bias=1e-9, lq=1e-9, force=1e-8)}


def _headline_args():
    return ["GAUSSIAN", 0.01, 0.005, 9.0, "PACE", 10, "TEMP", 300.0,
            "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "Q4", "STEINH", "L", 4, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18, "SW_FUNC_r", "ST",
            "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18, "SW_FUNC_r", "ST",
            "SYMBOL", "v1", "Q4.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID",
            "CV_dim", 2, "DIM", 1, 0, 1, 200, "v1", "DIM", 2, 0, 1, 200, "v2", "WT", 1]


@pytest.fixture(scope="module")
def headline():
    x, L = systems.config2(seed=2024)
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 2025, c), L)) for c in range(2)]
    st = O.make_sw("STEP", r0=3.9)
    orc = []
    for xc in xs:
        orc.append((O.steinh_l(4, xc, L, 3.9, st), O.steinh_l(6, xc, L, 3.9, st)))
    off, nbr = O.local_lists(xs[0], L, 3.9, st)
    return xs, L, orc, (off, nbr)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_headline_deck_256k_against_fp64_oracle(headline, precision):
    xs, L, orc, (off, nbr) = headline
    n = xs[0].shape[0]
    assert n == 256000
    m = mtd.Metad(_headline_args(), precision=precision)
    m.set_box([0, 0, 0], L)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, KB, True)
    tol = TOL[precision]
    report = {"precision": precision, "atoms": n}
    for k, step in enumerate([0, 1]):   # step 0 deposits (PACE 10), step 1 does not
        x = xs[k]
        o4, o6 = orc[k]
        f = np.zeros_like(x)
        m.post_force(step, x, f)
        s = np.array([o4["cv"], o6["cv"]])
        if step % 10 == 0:
            g.add_hill(s)
        V, dV = g.value(s)
        fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
        cv_err = [abs(m.cv[d] - s[d]) / abs(s[d]) for d in range(2)]
        bias_err = abs(m.compute_scalar() - V) / abs(V)
        fmax = np.abs(fo).max()
        force_err = float(np.abs(f - fo).max() / fmax)
        force_rms = float(np.sqrt(np.mean((f - fo) ** 2)) / fmax)
        lq_err = [H.rel(m.extract("Q%d.stein_q" % l, n), o["LQ"]) for l, o in ((4, o4), (6, o6))]
        report["step%d" % step] = dict(cv_rel=cv_err, bias_rel=bias_err, force_rel_max=force_err,
                                       force_rel_rms=force_rms, lq_rel_max=lq_err)
        assert max(cv_err) < tol["cv"], cv_err
        assert bias_err < tol["bias"], bias_err
        assert max(lq_err) < tol["lq"], lq_err
        assert force_err < tol["force"], force_err
        # neighbour counts and lists, per atom, exactly (both orders share one list)
        cnt = m.extract("Q4.nnb", n).astype(np.int32)
        assert np.array_equal(cnt, o4["nnb"]) and np.array_equal(cnt, o6["nnb"])
        if k == 0:
            counts, lists = m.neighbors("Q6", n, max_per_atom=int(cnt.max()))
            assert np.array_equal(counts, np.diff(off))
            assert np.array_equal(lists[lists >= 0], nbr)
    print("headline parity:", json.dumps(report))
    m.close()


def test_config1_full_protocol():
    x0, L = systems.config1()
    n = x0.shape[0]
    args = H.fix_args_q(l=6, rc=3.9, cap=18, sigma=0.01, h=0.005, biasf=10.0, pace=10, wt=0, nbins=1000)
    m = mtd.Metad(args, precision="fp64")
    m.set_box([0, 0, 0], L)
    g = O.Grid([[0.0, 1.0]], [1000], 0.01, 0.005, 10.0, 300.0, KB, False)
    worst = {"cv": 0.0, "bias": 0.0, "force": 0.0}
    hills = 0
    for step in range(1000):
        x = np.ascontiguousarray(systems.jitter(x0, 0.15, 2024, step))
        f = np.zeros_like(x)
        m.post_force(step, x, f)
        o = O.steinh_q(6, x, L, 3.9, 18, grad=(step % 50 == 0))
        if step % 10 == 0:
            g.add_hill([o["cv"]])
            hills += 1
        V, dV = g.value([o["cv"]])
        worst["cv"] = max(worst["cv"], abs(m.cv[0] - o["cv"]) / abs(o["cv"]))
        # relative to the largest bias so far: V(s) is ~0 where s is far from every hill
        worst["bias"] = max(worst["bias"], abs(m.compute_scalar() - V) / (0.005 * hills))
        if step % 50 == 0:
            fo = -dV[0] * o["grad"]
            err = H.rel(f, fo) if np.abs(fo).max() > 0 else float(np.abs(f).max())
            worst["force"] = max(worst["force"], err)
    grid = m.grid(1000)
    m.close()
    assert hills == 100
    assert worst["cv"] < 1e-12 and worst["bias"] < 1e-10 and worst["force"] < 1e-9, worst
    assert np.max(np.abs(grid - g.grid)) < 1e-12 * np.max(np.abs(g.grid))
    print("config-1 protocol: 1000 steps, %d hills, worst relative errors %s" % (hills, worst))
