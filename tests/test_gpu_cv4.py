"""CV_dim 4 through `fix metad` (hill-list bias): Q4.MEAN_SOLID, Q6.MEAN_SOLID,
the local-Q6 fraction above 0.5 (FERMI switch) and the k-vector S(k), with
WT hills kept as a list; V and dV/ds from the exact FP64 hill sum, or from the
learned bias when NN_BIAS 1 and its validation passes.  FP64 mode against the
FP64 oracle: 1e-9 relative on CVs and bias, 1e-8 on forces."""
import numpy as np
import pytest

import helpers as H
import mlp_oracle as MO
import oracle as O
import systems

pytestmark = pytest.mark.gpu

KB, TEMP, BIASF, H0, SIGMA = 8.617343e-5, 300.0, 10.0, 0.01, 0.05


def _args(extra=()):
    return (["GAUSSIAN", SIGMA, H0, BIASF, "PACE", 2, "TEMP", TEMP,
             "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
             "CAL", "NAME", "FE", "SW_FUNC", "FERMI", "r_0", 0.5, "alpha", 20.0,
             "CAL", "NAME", "Q4", "STEINH", "L", 4, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
             "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
             "CAL", "NAME", "Q6B", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
             "CAL", "NAME", "SK", "STRU_FACTOR_K", "all", "nk", 24, "kmag", systems.KMAG_111, "seed", 3,
             "SYMBOL", "v1", "Q4.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID",
             "SYMBOL", "v3", "Q6B.FRAC.FE", "SYMBOL", "v4", "SK.AVE",
             "CV_dim", 4, "DIM", 1, 0, 1, 10, "v1", "DIM", 2, 0, 1, 10, "v2", "DIM", 3, 0, 1, 10, "v3",
             "DIM", 4, 0, 2, 10, "v4", "WT", 1] + list(extra))


def _system():
    x, L = systems.small_slab(seed=41, nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    return np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 42), L)), L


def _oracle_cvs(x, L):
    st = O.make_sw("STEP", r0=3.9)
    fe = O.make_sw("FERMI", r0=0.5, alpha=20.0)
    o4 = O.steinh_l(4, x, L, 3.9, st, 1e-6, None, "MEAN_SOLID")
    o6 = O.steinh_l(6, x, L, 3.9, st, 1e-6, None, "MEAN_SOLID")
    o6f = O.steinh_l(6, x, L, 3.9, st, 1e-6, fe, "FRAC")
    sk = O.sk(x, systems.kvectors(24, systems.KMAG_111, 3))
    return [o4, o6, o6f, sk]


def test_cv4_hill_list_matches_oracle():
    x, L = _system()
    steps = [0, 1, 2, 3]
    m, out = H.run_gpu(_args(), x, L, [(s, x) for s in steps], precision="fp64")
    ref = _oracle_cvs(x, L)
    s = np.array([o["cv"] for o in ref])
    hills_c, hills_h = [], []
    for i, step in enumerate(steps):
        if hills_c:
            V, dV = MO.hill_sum(s[None, :], np.array(hills_c), np.array(hills_h), np.full(len(hills_h), SIGMA))
            V, dV = V[0], dV[0]
        else:
            V, dV = 0.0, np.zeros(4)
        if step % 2 == 0:
            w = H0 * np.exp(-V / (KB * TEMP * (BIASF - 1.0)))
            hills_c.append(s.copy())
            hills_h.append(w)
            V += w                       # the new hill: full height, no slope at its centre
        cv, bias, f, _ = out[i]
        assert H.rel(cv, s) < 1e-9
        assert H.rel(bias, V) < 1e-9
        fo = -sum(dV[d] * ref[d]["grad"] for d in range(4))
        assert H.rel(f, fo) < 1e-8


def test_cv4_learned_bias_falls_back_to_the_exact_sum():
    """NN_BIAS 1 with a tolerance no fit can meet: the network is refitted
    every 2 hills but never trusted, so every step equals the exact path."""
    x, L = _system()
    steps = [(s, x) for s in range(6)]
    _, exact = H.run_gpu(_args(), x, L, steps, precision="fp64")
    _, nn = H.run_gpu(_args(["NN_BIAS", 1, "NN_TOL", 1e-14, "NN_REFIT", 2, "NN_ITERS", 50]), x, L, steps,
                      precision="fp64")
    for (cv1, b1, f1, _), (cv2, b2, f2, _) in zip(exact, nn):
        assert np.array_equal(cv1, cv2) and b1 == b2 and np.array_equal(f1, f2)


def test_cv4_learned_bias_used_after_a_passing_fit(tmp_path):
    """With a tolerance the fit passes, the steps after a refit use the
    network plus the exact sum over the hills deposited since the fit.  The
    same fits replayed on a standalone learned-bias object (same seeds, same
    hills read back from HILLS) give the context's bias."""
    import mtd

    x, L = _system()
    path = str(tmp_path / "HILLS")
    m = mtd.Metad(_args(["NN_BIAS", 1, "NN_TOL", 1.0, "NN_REFIT", 2, "NN_ITERS", 300]), precision="fp64",
                  hills_path=path)
    m.set_box([0, 0, 0], L)
    bias = []
    for step in range(8):
        f = np.zeros_like(x)
        m.post_force(step, x, f)
        bias.append(m.compute_scalar())
        cv = m.cv.copy()
    assert m.nn_state() == (4, 4, True)
    m.close()
    rows = np.array([[float(v) for v in l.split()] for l in open(path) if not l.startswith("#")])
    c, w, sg = rows[:, 1:5], rows[:, 5], rows[:, 6]
    lo, hi = np.array([0.0, 0.0, 0.0, 0.0]), np.array([1.0, 1.0, 1.0, 2.0])
    nb = mtd.NNBias(lo, hi, seed=12345)
    nb.add_hills(c[:2], w[:2], sg[:2])
    nb.fit(ntrain=65536, iters=300, batch=4096, lr=2e-3, seed=1000 + 2)
    v1 = nb.eval(cv[None, :])[0][0]
    nb.add_hills(c[2:], w[2:], sg[2:])
    nb.fit(ntrain=65536, iters=300, batch=4096, lr=2e-3, seed=1000 + 4)
    v2 = nb.eval(cv[None, :])[0][0]
    nb.close()
    e3 = MO.hill_sum(cv[None, :], c[2:3], w[2:3], sg[2:3])[0][0]
    tol = 1e-5 * max(abs(v1), abs(v2), 1e-3)
    assert abs(bias[3] - v1) <= tol                  # fitted on hills 0, 2; none since
    assert abs(bias[5] - (v1 + e3)) <= tol           # plus the hill of step 4, exactly
    assert abs(bias[7] - v2) <= tol                  # refitted on all four
