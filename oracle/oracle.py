"""CPU FP64 oracle for the Metad-toy metadynamics hot path (TEST INFRASTRUCTURE ONLY).

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may
import this module; the product under ``metad-toy_b200/`` never does.

It wraps ``oracle/liboracle.so`` (a C restatement of the reference algorithm,
see mtd_oracle.h for the file:line each routine follows) and, where it was
built, ``oracle/_ref/libmtdref.so`` (the reference's own spherical-harmonic
header compiled for the host).  It also restates, in Python, the per-step
orchestration of ``FixMetadynamics::post_force``
(src/core/fix_crystallize.cu:386-472) and the DIM expression layer
(src/grids/DimSet.cu:28-97).
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

SW_TYPES = {"LINE": 0, "STEP": 1, "FERMI": 2, "TANH": 3, "RATIONAL": 4}


class Sw(C.Structure):
    _fields_ = [("type", C.c_int), ("r0", C.c_double), ("d0", C.c_double),
                ("alpha", C.c_double), ("n", C.c_int), ("m", C.c_int)]


class Box(C.Structure):
    _fields_ = [("L", C.c_double * 3), ("periodic", C.c_int * 3)]


def make_sw(kind="LINE", r0=None, d0=0.0, alpha=None, n=6, m=12):
    """Switching function with the defaults of zqc_switch_function.h:81-116."""
    t = SW_TYPES[kind]
    if r0 is None:
        r0 = 1.25 if kind == "RATIONAL" else (0.0 if kind == "LINE" else 1.0)
    if alpha is None:
        alpha = 20.0 if kind != "LINE" else 0.0
    return Sw(t, float(r0), float(d0), float(alpha), int(n), int(m))


def make_box(L, periodic=(1, 1, 1)):
    b = Box()
    for c in range(3):
        b.L[c] = float(L[c])
        b.periodic[c] = int(periodic[c])
    return b


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            subprocess.check_call(["make", "-s", "-C", HERE])
        L = C.CDLL(path)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        L.orc_sw_f.restype = C.c_double
        L.orc_sw_f.argtypes = [C.POINTER(Sw), C.c_double]
        L.orc_sw_df.restype = C.c_double
        L.orc_sw_df.argtypes = [C.POINTER(Sw), C.c_double]
        L.orc_sw_invert_for_eps.restype = C.c_double
        L.orc_sw_invert_for_eps.argtypes = [C.POINTER(Sw), C.c_double]
        L.orc_minimg.argtypes = [C.POINTER(Box), dp, dp, dp]
        L.orc_ylm.argtypes = [C.c_int, dp, dp, dp]
        L.orc_ylm_grad.argtypes = [C.c_int, dp, dp, dp, dp, dp]
        L.orc_steinh_q.argtypes = [C.c_int, C.c_int, dp, C.POINTER(Box), ip, C.c_double, C.c_int,
                                   C.c_int, C.POINTER(Sw), dp, dp, ip, ip, ip, dp, dp]
        L.orc_steinh_l.argtypes = [C.c_int, C.c_int, dp, C.POINTER(Box), ip, C.c_double, C.POINTER(Sw),
                                   C.c_double, C.POINTER(Sw), C.c_int, dp, dp, dp, dp, ip, dp, dp, dp]
        L.orc_debye.argtypes = [C.c_int, dp, C.POINTER(Box), ip, C.c_double, C.c_double, C.c_int,
                                C.POINTER(Sw), dp, dp, dp]
        L.orc_debye_w.argtypes = [C.c_int, dp, C.POINTER(Box), ip, C.c_double, C.c_double, C.c_int,
                                  C.POINTER(Sw), dp, dp, dp, dp]
        L.orc_sk.argtypes = [C.c_int, dp, ip, C.c_int, dp, dp, dp, dp, dp]
        L.orc_grid_deposit.argtypes = [C.c_int, ip, dp, dp, dp, C.c_double, C.c_double, C.c_double]
        L.orc_grid_value.restype = C.c_double
        L.orc_grid_value.argtypes = [C.c_int, ip, dp, dp, dp, dp]
        L.orc_hill_sum.argtypes = [C.c_int, C.c_int, dp, dp, dp, C.c_int, dp, dp, dp]
        i64pp, ipp = C.POINTER(C.POINTER(C.c_int64)), C.POINTER(C.POINTER(C.c_int))
        L.orc_pairs.argtypes = [C.c_int, dp, C.POINTER(Box), C.c_double, i64pp, ipp]
        L.orc_local_lists.argtypes = [C.c_int, dp, C.POINTER(Box), C.c_double, C.POINTER(Sw), C.c_double, i64pp, ipp]
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_get_threads.restype = C.c_int
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's Y_lm header compiled for the host, or None if it was not built."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libmtdref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
        R.ref_ylm.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, dp]
        R.ref_dylm.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, dp]
        R.ref_q_grad_faithful.argtypes = [C.c_int, C.c_int, C.c_int, ip, ip, dp, dp, dp, ip, C.c_int, dp]
        _REF = R
    return _REF


def set_threads(n):
    lib().orc_set_threads(int(n))


def get_threads():
    return lib().orc_get_threads()


# --------------------------------------------------------------------------------------
# Thin wrappers
# --------------------------------------------------------------------------------------
def sw_f(sw, x):
    return lib().orc_sw_f(C.byref(sw), float(x))


def sw_df(sw, x):
    return lib().orc_sw_df(C.byref(sw), float(x))


def sw_invert_for_eps(sw, eps):
    return lib().orc_sw_invert_for_eps(C.byref(sw), float(eps))


def ylm(l, d):
    d = np.ascontiguousarray(d, dtype=np.float64)
    re = np.zeros(l + 1)
    im = np.zeros(l + 1)
    lib().orc_ylm(l, _dp(d), _dp(re), _dp(im))
    return re + 1j * im


def ylm_grad(l, d):
    d = np.ascontiguousarray(d, dtype=np.float64)
    re, im = np.zeros(l + 1), np.zeros(l + 1)
    gre, gim = np.zeros(3 * (l + 1)), np.zeros(3 * (l + 1))
    lib().orc_ylm_grad(l, _dp(d), _dp(re), _dp(im), _dp(gre), _dp(gim))
    return re + 1j * im, (gre + 1j * gim).reshape(l + 1, 3)


def _group(n, ingroup):
    if ingroup is None:
        return np.ones(n, dtype=np.int32)
    return np.ascontiguousarray(ingroup, dtype=np.int32)


def steinh_q(l, x, L, rc, cap, mode="AVE", swcv=None, ingroup=None, periodic=(1, 1, 1), grad=True):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    g = _group(n, ingroup)
    S = 2 * (l + 1)
    Q = np.zeros(n)
    qlm = np.zeros(n * S)
    nk = np.zeros(n, np.int32)
    nrc = np.zeros(n, np.int32)
    kept = np.zeros(n * cap, np.int32)
    cv = np.zeros(1)
    gr = np.zeros(3 * n) if grad else None
    sw = swcv if swcv is not None else make_sw("LINE")
    box = make_box(L, periodic)
    rc_ = lib().orc_steinh_q(l, n, _dp(x), C.byref(box), _ip(g), float(rc), int(cap),
                             0 if mode == "AVE" else 1, C.byref(sw), _dp(Q), _dp(qlm), _ip(nk), _ip(nrc),
                             _ip(kept), _dp(cv), _dp(gr) if grad else None)
    assert rc_ == 0
    out = dict(Q=Q, qlm=qlm.reshape(n, S), nkept=nk, nrc=nrc, kept=kept.reshape(n, cap), cv=cv[0])
    if grad:
        out["grad"] = gr.reshape(n, 3)
    return out


def _csr(fn, n, *args):
    off, nbr = C.POINTER(C.c_int64)(), C.POINTER(C.c_int)()
    fn(*args, C.byref(off), C.byref(nbr))
    o = np.ctypeslib.as_array(off, shape=(n + 1,)).copy()
    m = int(o[-1])
    v = np.ctypeslib.as_array(nbr, shape=(max(m, 1),))[:m].copy()
    lib().orc_free(C.cast(off, C.c_void_p))
    lib().orc_free(C.cast(nbr, C.c_void_p))
    return o, v


def pairs(x, L, rcut, periodic=(1, 1, 1)):
    """All ordered pairs (i, j != i) with r2 <= rcut^2: CSR (off[n+1], nbr), j ascending."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    box = make_box(L, periodic)
    return _csr(lib().orc_pairs, x.shape[0], x.shape[0], _dp(x), C.byref(box), float(rcut))


def local_lists(x, L, rlist, swr, eps=1e-6, periodic=(1, 1, 1)):
    """The neighbour lists of steinh_l (r <= rlist, sigma(r) >= eps): CSR, j ascending."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    box = make_box(L, periodic)
    return _csr(lib().orc_local_lists, x.shape[0], x.shape[0], _dp(x), C.byref(box), float(rlist), C.byref(swr),
                float(eps))


LOCAL_MODES = {"MEAN_SOLID": 0, "AVE": 0, "NSOLID": 1, "SW_FUNC": 1, "FRAC": 2}


def steinh_l(l, x, L, rlist, swr, eps=1e-6, swcv=None, mode="MEAN_SOLID", ingroup=None,
             periodic=(1, 1, 1), grad=True):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    g = _group(n, ingroup)
    S = 2 * (l + 1)
    LQ, NF = np.zeros(n), np.zeros(n)
    LQlm, qlm = np.zeros(n * S), np.zeros(n * S)
    nnb = np.zeros(n, np.int32)
    cv, sums = np.zeros(1), np.zeros(3)
    gr = np.zeros(3 * n) if grad else None
    sw = swcv if swcv is not None else make_sw("LINE")
    box = make_box(L, periodic)
    rc_ = lib().orc_steinh_l(l, n, _dp(x), C.byref(box), _ip(g), float(rlist), C.byref(swr), float(eps),
                             C.byref(sw), LOCAL_MODES[mode], _dp(LQ), _dp(LQlm), _dp(qlm), _dp(NF), _ip(nnb),
                             _dp(cv), _dp(sums), _dp(gr) if grad else None)
    assert rc_ == 0
    out = dict(LQ=LQ, LQlm=LQlm.reshape(n, S), qlm=qlm.reshape(n, S), NF=NF, nnb=nnb, cv=cv[0], sums=sums)
    if grad:
        out["grad"] = gr.reshape(n, 3)
    return out


def chem_type_weights(types, ctarget=0.0, sigma=1.0, cmap=None):
    """Per-atom STRU_FACTOR Chemical weights: Chem_map value of the atom's type,
    else exp(-(type - ctarget)^2 / (2 sigma^2)); type 0 weighs 0
    (Stru_fact_chem_env constructor, src/cvs/CVs_Strufactor_chem.cu:33-55)."""
    cmap = dict(cmap or {})
    t = np.asarray(types, dtype=np.int64)
    w = np.exp(-(t - ctarget) ** 2 / (2.0 * sigma ** 2))
    for k, v in cmap.items():
        w[t == k] = v
    w[t == 0] = 0.0
    return np.ascontiguousarray(w, dtype=np.float64)


def debye(x, L, rc, qf, mode="AVE", sw=None, ingroup=None, periodic=(1, 1, 1), grad=True, weights=None):
    x = np.ascontiguousarray(x, dtype=np.float64)
    n = x.shape[0]
    g = _group(n, ingroup)
    S = np.zeros(n)
    cv = np.zeros(1)
    gr = np.zeros(3 * n) if grad else None
    s = sw if sw is not None else make_sw("LINE")
    box = make_box(L, periodic)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    lib().orc_debye_w(n, _dp(x), C.byref(box), _ip(g), float(rc), float(qf), 0 if mode == "AVE" else 1,
                      C.byref(s), _dp(w) if w is not None else None, _dp(S), _dp(cv), _dp(gr) if grad else None)
    out = dict(S=S, cv=cv[0])
    if grad:
        out["grad"] = gr.reshape(n, 3)
    return out


def sk(x, kvecs, ingroup=None, grad=True):
    x = np.ascontiguousarray(x, dtype=np.float64)
    k = np.ascontiguousarray(kvecs, dtype=np.float64)
    n, nk = x.shape[0], k.shape[0]
    g = _group(n, ingroup)
    rho, Sk, cv = np.zeros(2 * nk), np.zeros(nk), np.zeros(1)
    gr = np.zeros(3 * n) if grad else None
    lib().orc_sk(n, _dp(x), _ip(g), nk, _dp(k), _dp(rho), _dp(Sk), _dp(cv), _dp(gr) if grad else None)
    out = dict(rho=rho.reshape(nk, 2), Sk=Sk, cv=cv[0])
    if grad:
        out["grad"] = gr.reshape(n, 3)
    return out


def hill_sum(centers, heights, sigmas, points, grad=True):
    centers = np.ascontiguousarray(centers, dtype=np.float64)
    points = np.ascontiguousarray(points, dtype=np.float64)
    heights = np.ascontiguousarray(heights, dtype=np.float64)
    sigmas = np.ascontiguousarray(sigmas, dtype=np.float64)
    D = centers.shape[1]
    V = np.zeros(points.shape[0])
    dV = np.zeros(points.shape) if grad else None
    lib().orc_hill_sum(D, centers.shape[0], _dp(centers), _dp(heights), _dp(sigmas), points.shape[0],
                       _dp(points), _dp(V), _dp(dV) if grad else None)
    return (V, dV) if grad else V


class Grid:
    """Uniform bias grid, restating src/grids/GH_t0_uniformGrid.cu."""

    def __init__(self, bounds, nbins, sigma, height0, biasf, temp, kb, wt):
        self.D = len(nbins)
        self.nbin = np.ascontiguousarray(nbins, dtype=np.int32)
        self.bound = np.ascontiguousarray(np.asarray(bounds, dtype=np.float64).reshape(-1))
        self.grid = np.zeros(int(np.prod(nbins)))
        self.sigma, self.h0, self.biasf, self.temp, self.kb, self.wt = sigma, height0, biasf, temp, kb, wt

    def value(self, s):
        s = np.ascontiguousarray(s, dtype=np.float64)
        dV = np.zeros(self.D)
        V = lib().orc_grid_value(self.D, _ip(self.nbin), _dp(self.bound), _dp(self.grid), _dp(s), _dp(dV))
        return V, dV

    def deposit(self, s, w, sigma=None):
        s = np.ascontiguousarray(s, dtype=np.float64)
        sg = self.sigma if sigma is None else sigma
        lib().orc_grid_deposit(self.D, _ip(self.nbin), _dp(self.bound), _dp(self.grid), _dp(s), float(w),
                               float(sg), float(self.sigma))

    def add_hill(self, s):
        """add_hill (GH_t0_uniformGrid.cu:195-208): WT height from V before deposit."""
        V = self.value(s)[0] if self.wt else 0.0
        w = self.h0 * math.exp(-V / (self.temp * self.kb * (self.biasf - 1.0)))
        self.deposit(s, w)
        return w


# --------------------------------------------------------------------------------------
# DIM expressions: a small recursive-descent evaluator with forward-mode derivatives.
# It stands in for exprtk (third_party/exprtk.hpp) as used by src/grids/DimSet.cu:54-97;
# derivatives are exact instead of exprtk::derivative's central difference.
# --------------------------------------------------------------------------------------
class _Dual:
    __slots__ = ("v", "d")

    def __init__(self, v, d):
        self.v, self.d = v, d


_FUNCS1 = {
    "sin": (math.sin, math.cos), "cos": (math.cos, lambda x: -math.sin(x)),
    "exp": (math.exp, math.exp), "log": (math.log, lambda x: 1.0 / x),
    "sqrt": (math.sqrt, lambda x: 0.5 / math.sqrt(x)), "tanh": (math.tanh, lambda x: 1.0 - math.tanh(x) ** 2),
    "abs": (abs, lambda x: (1.0 if x > 0 else (-1.0 if x < 0 else 0.0))),
}


def eval_expr(expr, values):
    """Evaluate expression `expr` over symbol values dict -> (value, {sym: d/dsym})."""
    syms = list(values.keys())
    idx = {s: i for i, s in enumerate(syms)}
    toks = []
    i = 0
    while i < len(expr):
        ch = expr[i]
        if ch.isspace():
            i += 1
        elif ch.isdigit() or ch == ".":
            j = i
            while j < len(expr) and (expr[j].isdigit() or expr[j] in ".eE" or
                                     (expr[j] in "+-" and expr[j - 1] in "eE")):
                j += 1
            toks.append(("num", float(expr[i:j])))
            i = j
        elif ch.isalpha() or ch == "_":
            j = i
            while j < len(expr) and (expr[j].isalnum() or expr[j] == "_"):
                j += 1
            toks.append(("id", expr[i:j]))
            i = j
        else:
            toks.append(("op", ch))
            i += 1
    pos = [0]
    nd = len(syms)

    def peek():
        return toks[pos[0]] if pos[0] < len(toks) else ("end", None)

    def take():
        t = peek()
        pos[0] += 1
        return t

    def const(v):
        return _Dual(v, [0.0] * nd)

    def add(a, b, s=1.0):
        return _Dual(a.v + s * b.v, [x + s * y for x, y in zip(a.d, b.d)])

    def mul(a, b):
        return _Dual(a.v * b.v, [a.v * y + b.v * x for x, y in zip(a.d, b.d)])

    def div(a, b):
        return _Dual(a.v / b.v, [(x * b.v - a.v * y) / (b.v * b.v) for x, y in zip(a.d, b.d)])

    def pw(a, b):
        v = a.v ** b.v
        d = []
        for x, y in zip(a.d, b.d):
            t = b.v * a.v ** (b.v - 1) * x if x != 0.0 else 0.0
            if y != 0.0:
                t += v * math.log(a.v) * y
            d.append(t)
        return _Dual(v, d)

    def primary():
        t = take()
        if t[0] == "num":
            return const(t[1])
        if t[0] == "id":
            name = t[1]
            if peek() == ("op", "("):
                take()
                args = [expr_()]
                while peek() == ("op", ","):
                    take()
                    args.append(expr_())
                assert take() == ("op", ")")
                if name in _FUNCS1:
                    f, df = _FUNCS1[name]
                    a = args[0]
                    g = df(a.v)
                    return _Dual(f(a.v), [g * x for x in a.d])
                if name == "pow":
                    return pw(args[0], args[1])
                if name in ("min", "max"):
                    a, b = args
                    pick = (a.v <= b.v) if name == "min" else (a.v >= b.v)
                    return a if pick else b
                raise ValueError("unknown function " + name)
            if name == "pi":
                return const(math.pi)
            if name == "e" and name not in idx:
                return const(math.e)
            d = [0.0] * nd
            d[idx[name]] = 1.0
            return _Dual(values[name], d)
        if t == ("op", "("):
            v = expr_()
            assert take() == ("op", ")")
            return v
        raise ValueError("bad token %r" % (t,))

    def unary():
        # unary minus binds looser than '^':  -a^b = -(a^b),  a^-b = a^(-b)
        if peek() == ("op", "-"):
            take()
            v = unary()
            return _Dual(-v.v, [-x for x in v.d])
        if peek() == ("op", "+"):
            take()
            return unary()
        return power()

    def power():
        b = primary()
        if peek() == ("op", "^"):
            take()
            e = unary()
            return pw(b, e)
        return b

    def term():
        v = unary()
        while peek() in (("op", "*"), ("op", "/")):
            op = take()[1]
            r = unary()
            v = mul(v, r) if op == "*" else div(v, r)
        return v

    def expr_():
        v = term()
        while peek() in (("op", "+"), ("op", "-")):
            op = take()[1]
            r = term()
            v = add(v, r, 1.0 if op == "+" else -1.0)
        return v

    res = expr_()
    assert peek()[0] == "end", "trailing tokens in expression"
    return res.v, dict(zip(syms, res.d))
