"""Device-side parity for the CV variants: every one through a full step of
the C ABI (neighbour lists, values, reductions, DIM expressions, grid,
forces) against the FP64 oracle.

  * STEINH Q SW_FUNC value and gradient (src/cvs/CVs_Steinhardt.cu:961-1098,
    :1701-1863) with FERMI, TANH, LINE and RATIONAL (n = 2m branch) switches;
  * LINE, TANH and RATIONAL switching functions in a device step
    (include/utils/zqc_switch_function.h:163-313): RATIONAL 6/12, the general
    RATIONAL n/m branch and TANH as the STEINH L distance switch, TANH,
    RATIONAL n = 2m and LINE as its CV switch;
  * l = 3 (include/CVsets/CV_Steinhardt_math.h:981-1040), STEINH Q and the
    fused STEINH L pair (3, 6);
  * composite DIM expressions with their chain factors (src/grids/DimSet.cu:54-97);
  * the STEINH Q cutoff_Natoms cap where it binds, with exact r^2 ties on a
    perfect lattice: per-atom kept lists compared exactly
    (src/cvs/CVs_Steinhardt.cu:1324-1406).

Tolerances: FP64 mode 1e-9 relative on CVs and bias, 1e-8 on the largest
force component; mixed mode 2e-5 and 2e-3.  Neighbour counts and lists are
compared exactly.
"""
import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-9, 1e-8), "mixed": (2e-5, 2e-3)}
KB = 8.617343e-5


def _sw_args(name, kind, **kw):
    a = ["CAL", "NAME", name, "SW_FUNC", kind]
    for k in ("r_0", "d_0", "alpha", "n", "m"):
        if k in kw:
            a += [k, kw[k]]
    return a


def _sw_oracle(kind, **kw):
    return O.make_sw(kind, r0=kw.get("r_0"), d0=kw.get("d_0", 0.0), alpha=kw.get("alpha"), n=kw.get("n", 6),
                     m=kw.get("m", 12))


def _fcc_jittered(nc=6, seed=3, sigma=0.15):
    x, L = systems.fcc(nc, 5.26), np.array([nc * 5.26] * 3)
    return np.ascontiguousarray(systems.wrap(systems.jitter(x, sigma, seed), L)), L


def _step_and_compare(args, x, L, precision, cvs_o, grads_o, dims, wt, biasf=10.0, temp=300.0, sigma=0.01,
                      h0=0.005, expr_chain=None):
    """One deposit step on the GPU against the oracle: cvs_o / grads_o are the
    symbols' oracle values and gradients; expr_chain(v) -> (s, J) maps them to
    the DIM values and ds/dv (identity when None)."""
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    cv, bias, f, _ = out[0]
    v = np.asarray(cvs_o, dtype=np.float64)
    if expr_chain is None:
        s, J = v, np.eye(len(v))
    else:
        s, J = expr_chain(v)
    g = O.Grid([d[:2] for d in dims], [d[2] for d in dims], sigma, h0, biasf, temp, KB, wt)
    g.add_hill(s)
    V, dV = g.value(s)
    dVdv = J.T @ dV
    fo = -sum(dVdv[q] * grads_o[q] for q in range(len(v)))
    tcv, tf = TOL[precision]
    assert H.rel(cv, s) < tcv, (cv, s)
    # relative to the hill height: V(s) is ~0 where s sits in a hill's tail (s near a grid edge)
    assert abs(bias - V) < max(tcv, 1e-12) * max(abs(V), h0), (bias, V)
    assert H.rel(f, fo) < tf, H.rel(f, fo)
    return m


# ------------------------------------------------------------------ STEINH Q SW_FUNC
Q_SWITCHES = {
    "fermi": ("FERMI", dict(r_0=0.45, alpha=20.0)),
    "tanh": ("TANH", dict(r_0=0.47, alpha=15.0)),
    "rational_n_2m": ("RATIONAL", dict(r_0=0.8, d_0=0.1, n=4, m=2)),
    "line": ("LINE", dict()),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("sw", list(Q_SWITCHES))
def test_steinh_q_sw_func(sw, precision):
    x, L = _fcc_jittered()
    n = x.shape[0]
    kind, kw = Q_SWITCHES[sw]
    # Sum f(Q) is of order n: the DIM expression maps it onto [0, 1] so that one
    # isotropic hill width serves both axes
    hi = 2.0 * n
    args = (["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 10] + _sw_args("SWC", kind, **kw) +
            ["CAL", "NAME", "Q6", "STEINH", "Q", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18,
             "SYMBOL", "v1", "Q6.SW_FUNC.SWC", "SYMBOL", "v2", "Q6.AVE", "CV_dim", 2,
             "DIM", 1, 0.0, 1.0, 400, "v1/%r" % hi, "DIM", 2, 0.0, 1.0, 200, "v2", "WT", 1])
    swc = _sw_oracle(kind, **kw)
    o_sw = O.steinh_q(6, x, L, 3.9, 18, mode="SW_FUNC", swcv=swc)
    o_av = O.steinh_q(6, x, L, 3.9, 18)
    assert o_sw["cv"] == pytest.approx(sum(O.sw_f(swc, q) for q in o_av["Q"]), rel=1e-12)
    _step_and_compare(args, x, L, precision, [o_sw["cv"], o_av["cv"]], [o_sw["grad"], o_av["grad"]],
                      [[0.0, 1.0, 400], [0.0, 1.0, 200]], True, sigma=0.01,
                      expr_chain=lambda v: (np.array([v[0] / hi, v[1]]), np.diag([1.0 / hi, 1.0])))


# ------------------------------------------------------------------ STEINH L switching functions
L_CASES = {
    # name: (SW_FUNC_r, cv switch (or None), mode)
    "r_tanh__cv_tanh_mean": (("TANH", dict(r_0=3.5, alpha=-8.0)), ("TANH", dict(r_0=0.35, alpha=20.0)),
                             "MEAN_SOLID"),
    "r_rational612__cv_line_mean": (("RATIONAL", dict(r_0=0.3, d_0=3.2, n=6, m=12)), ("LINE", dict()),
                                    "MEAN_SOLID"),
    "r_rational_general__cv_rational_n2m_nsolid": (("RATIONAL", dict(r_0=0.3, d_0=3.3, n=8, m=14)),
                                                    ("RATIONAL", dict(r_0=0.5, d_0=0.0, n=4, m=2)), "NSOLID"),
    "r_fermi__cv_tanh_frac": (("FERMI", dict(r_0=3.9, alpha=-8.0)), ("TANH", dict(r_0=0.35, alpha=20.0)),
                              "FRAC"),
}


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", list(L_CASES))
def test_steinh_l_switching_functions(case, precision):
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 7), L))
    n = x.shape[0]
    (rk, rkw), (ck, ckw), mode = L_CASES[case]
    swr, swc = _sw_oracle(rk, **rkw), _sw_oracle(ck, **ckw)
    rl = O.sw_invert_for_eps(swr, 1e-6)
    o4 = O.steinh_l(4, x, L, rl, swr, 1e-6, swc, mode)
    o6 = O.steinh_l(6, x, L, rl, swr, 1e-6, swc, mode)
    # the DIMs scale both CVs into the middle of the grid, where V and dV/ds
    # are of the hill's size (outside it they are a hill's far tail)
    scale = float(2.5 * max(abs(o4["cv"]), abs(o6["cv"])))
    args = (["GAUSSIAN", 0.01, 0.005, 9.0, "PACE", 10, "TEMP", 300.0] + _sw_args("SWR", rk, **rkw) +
            _sw_args("SWC", ck, **ckw))
    for l in (4, 6):
        args += ["CAL", "NAME", "Q%d" % l, "STEINH", "L", l, "all", "SW_FUNC_r", "SWR"]
    args += ["SYMBOL", "v1", "Q4.%s.SWC" % mode, "SYMBOL", "v2", "Q6.%s.SWC" % mode, "CV_dim", 2,
             "DIM", 1, 0.0, 1.0, 100, "v1/%r" % scale, "DIM", 2, 0.0, 1.0, 100, "v2/%r" % scale,
             "WT", 1]
    c = 1.0 / scale
    m = _step_and_compare(args, x, L, precision, [o4["cv"], o6["cv"]], [o4["grad"], o6["grad"]],
                          [[0.0, 1.0, 100], [0.0, 1.0, 100]], True, biasf=9.0,
                          expr_chain=lambda v: (v * c, np.diag([c, c])))
    counts, lists = m.neighbors("Q4", n, max_per_atom=int(o4["nnb"].max()))
    off, nbr = O.local_lists(x, L, rl, swr, 1e-6)
    assert np.array_equal(counts, np.diff(off)) and np.array_equal(counts, o4["nnb"])
    assert np.array_equal(lists[lists >= 0], nbr)
    m.close()


# ------------------------------------------------------------------ l = 3
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_l3_steinh_q_and_fused_local_pair(precision):
    x, L = _fcc_jittered(nc=5, seed=9)
    args = ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "Q3", "STEINH", "Q", 3, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18,
            "SYMBOL", "v1", "Q3.AVE", "CV_dim", 1, "DIM", 1, 0.0, 1.0, 1000, "v1", "WT", 0]
    o = O.steinh_q(3, x, L, 3.9, 18)
    m = _step_and_compare(args, x, L, precision, [o["cv"]], [o["grad"]], [[0.0, 1.0, 1000]], False)
    assert H.rel(m.extract("Q3.stein_q", x.shape[0]), o["Q"]) < TOL[precision][0] * 10
    m.close()
    xs, Ls = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    xs = np.ascontiguousarray(systems.wrap(systems.jitter(xs, 0.05, 11), Ls))
    args = ["GAUSSIAN", 0.01, 0.005, 9.0, "PACE", 10, "TEMP", 300.0,
            "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "Q3", "STEINH", "L", 3, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "SYMBOL", "v1", "Q3.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID", "CV_dim", 2,
            "DIM", 1, 0.0, 1.0, 200, "v1", "DIM", 2, 0.0, 1.0, 200, "v2", "WT", 1]
    st = O.make_sw("STEP", r0=3.9)
    o3, o6 = O.steinh_l(3, xs, Ls, 3.9, st), O.steinh_l(6, xs, Ls, 3.9, st)
    m = _step_and_compare(args, xs, Ls, precision, [o3["cv"], o6["cv"]], [o3["grad"], o6["grad"]],
                          [[0.0, 1.0, 200], [0.0, 1.0, 200]], True, biasf=9.0)
    assert H.rel(m.extract("Q3.stein_q", xs.shape[0]), o3["LQ"]) < TOL[precision][0] * 10
    m.close()


# ------------------------------------------------------------------ composite DIM expressions
EXPRS = {
    "mean_and_product": (["(v1+v2)/2", "v1*v2"],
                         lambda v: (np.array([(v[0] + v[1]) / 2, v[0] * v[1]]),
                                    np.array([[0.5, 0.5], [v[1], v[0]]]))),
    "functions": (["sqrt(v1^2+v2^2)/2", "exp(-v1)*v2"],
                  lambda v: (np.array([np.hypot(v[0], v[1]) / 2, np.exp(-v[0]) * v[1]]),
                             np.array([[v[0] / (2 * np.hypot(v[0], v[1])), v[1] / (2 * np.hypot(v[0], v[1]))],
                                       [-np.exp(-v[0]) * v[1], np.exp(-v[0])]]))),
}


def _oracle_chain(exprs):
    """s(v) and ds/dv from the oracle's expression evaluator (pinned to exprtk's
    own outputs by tests/test_expr_exprtk.py)."""
    def chain(v):
        res = [O.eval_expr(e, {"v1": float(v[0]), "v2": float(v[1])}) for e in exprs]
        return np.array([r[0] for r in res]), np.array([[r[1]["v1"], r[1]["v2"]] for r in res])
    return chain


# exprtk operators beyond arithmetic inside a device step: selection,
# comparison, logic, clamp, variadic functions, implicit multiplication
for _name, _exprs in {
        "selection_and_clamp": ["v1 > v2 ? v1 : 0.5(v1 + v2)", "clamp(0.05, 1.3*v2 - 0.1, 0.95)"],
        "logic_and_variadic": ["avg(v1, v2, v1 v2) + 0.1*(v1 < v2 and v2 > 0)",
                               "min(v1, v2, 0.9) + if(v2 > 0.3, 0.05 sin(v1), 0)"]}.items():
    EXPRS[_name] = (_exprs, _oracle_chain(_exprs))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", list(EXPRS))
def test_composite_dim_expressions(case, precision):
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 13), L))
    exprs, chain = EXPRS[case]
    args = H.fix_args_local()
    i = args.index("DIM")
    args = args[:i] + ["DIM", 1, 0.0, 1.0, 200, exprs[0], "DIM", 2, 0.0, 1.0, 200, exprs[1], "WT", 1]
    o4, o6 = H.oracle_local(x, L, 4), H.oracle_local(x, L, 6)
    v = np.array([o4["cv"], o6["cv"]])
    for d, e in enumerate(exprs):   # the oracle's expression evaluator agrees with the closed forms
        val, der = O.eval_expr(e, {"v1": v[0], "v2": v[1]})
        s, J = chain(v)
        assert val == pytest.approx(s[d], rel=1e-14) and [der["v1"], der["v2"]] == pytest.approx(J[d], rel=1e-12)
    m = _step_and_compare(args, x, L, precision, list(v), [o4["grad"], o6["grad"]],
                          [[0.0, 1.0, 200], [0.0, 1.0, 200]], True, biasf=9.0, expr_chain=chain)
    m.close()


# ------------------------------------------------------------------ cutoff_Natoms where it binds
def _tie_count(x, L, rc, cap):
    """Atoms whose cap-th and (cap+1)-th nearest neighbours lie at bitwise equal
    r^2 (the FP64 minimum-image operations of the oracle, in numpy)."""
    n = x.shape[0]
    ties = 0
    for i in range(n):
        d = x - x[i]
        d -= L * np.rint(d / L)
        r2 = (d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2]
        r2 = np.sort(r2[(r2 <= rc * rc) & (r2 >= 1e-12)])
        if r2.size > cap and r2[cap - 1] == r2[cap]:
            ties += 1
    return ties


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("deck", ["perfect_fcc_rc5.5_cap14", "jittered_fcc_rc4.3_cap8"])
def test_cap_binds_with_exact_ties(deck, precision):
    if deck.startswith("perfect"):
        x, L = systems.fcc(5, 5.26), np.array([5 * 5.26] * 3)
        x = np.ascontiguousarray(x)
        rc, cap = 5.5, 14
        # the second shell's six are tied in exact FP64 arithmetic for most atoms
        # (rounding separates the rest by an ulp): 236 of the 500 atoms here
        assert _tie_count(x, L, rc, cap) > x.shape[0] // 3
    else:
        x, L = _fcc_jittered(nc=5, seed=15, sigma=0.12)
        rc, cap = 4.3, 8
    n = x.shape[0]
    args = H.fix_args_q(rc=rc, cap=cap)
    o = O.steinh_q(6, x, L, rc, cap)
    assert np.all(o["nrc"] > cap)   # the cap binds for every atom
    m = _step_and_compare(args, x, L, precision, [o["cv"]], [o["grad"]], [[0.0, 1.0, 1000]], False)
    counts, lists = m.neighbors("Q6", n, max_per_atom=cap)
    assert np.array_equal(counts, o["nkept"])
    assert np.array_equal(m.extract("Q6.nnb", n).astype(np.int32), o["nkept"])
    assert np.array_equal(m.extract("Q6.nrc", n).astype(np.int32), o["nrc"])
    assert np.array_equal(lists, np.sort(o["kept"], axis=1))
    assert H.rel(m.extract("Q6.stein_q", n), o["Q"]) < TOL[precision][0] * 10
    m.close()
