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
        self.v, self.d = float(v), d


def _np(f):
    def g(*a):
        with np.errstate(all="ignore"):
            return float(f(*[np.float64(x) for x in a]))
    return g


_sin, _cos, _tan, _exp, _log, _sqrt = (_np(np.sin), _np(np.cos), _np(np.tan), _np(np.exp), _np(np.log),
                                       _np(np.sqrt))
_pow, _floor, _ceil, _trunc, _fmod = _np(np.power), _np(np.floor), _np(np.ceil), _np(np.trunc), _np(np.fmod)


def _erf(x):
    return math.erf(x) if math.isfinite(x) else (math.copysign(1.0, x) if not math.isnan(x) else math.nan)


def _erfc(x):
    return 1.0 - _erf(x) if not math.isfinite(x) else math.erfc(x)


def _round(v):   # exprtk round_impl: half away from zero through floor / ceil
    return _ceil(v - 0.5) if v < 0 else _floor(v + 0.5)


def _sinc(x):
    return (_sin(x) / x, (_cos(x) - _sin(x) / x) / x) if abs(x) >= 2.220446049250313e-16 else (1.0, 0.0)


def _root(x, n):
    if x < 0:
        odd = n == _trunc(n) and _fmod(n, 2.0) != 0.0
        v = -_pow(-x, 1.0 / n) if odd else math.nan
    else:
        v = _pow(x, 1.0 / n)
    with np.errstate(all="ignore"):
        dx = float(np.float64(v) / (np.float64(n) * np.float64(x)))
    dn = -v * _log(abs(x)) / (n * n) if x != 0 else 0.0
    return v, dx, dn


def _near(a, b):   # exprtk equal(): within 1e-10 of max(1, |a|, |b|)
    return abs(a - b) <= max(1.0, abs(a), abs(b)) * 1e-10


_PI = math.pi
# name -> (value(x), d value / dx)
_FUNCS1 = {
    "sin": (_sin, _cos), "cos": (_cos, lambda x: -_sin(x)), "tan": (_tan, lambda x: 1.0 + _tan(x) ** 2),
    "asin": (_np(np.arcsin), lambda x: 1.0 / _sqrt(1.0 - x * x)),
    "acos": (_np(np.arccos), lambda x: -1.0 / _sqrt(1.0 - x * x)),
    "atan": (_np(np.arctan), lambda x: 1.0 / (1.0 + x * x)),
    "exp": (_exp, _exp), "log": (_log, lambda x: 1.0 / x),
    "log10": (_np(np.log10), lambda x: 1.0 / (x * math.log(10.0))),
    "log2": (_np(np.log2), lambda x: 1.0 / (x * math.log(2.0))),
    "log1p": (_np(np.log1p), lambda x: 1.0 / (1.0 + x)), "expm1": (_np(np.expm1), _exp),
    "sqrt": (_sqrt, lambda x: 0.5 / _sqrt(x)),
    "abs": (abs, lambda x: (1.0 if x > 0 else (-1.0 if x < 0 else 0.0))),
    "tanh": (_np(np.tanh), lambda x: 1.0 - _np(np.tanh)(x) ** 2),
    "sinh": (_np(np.sinh), _np(np.cosh)), "cosh": (_np(np.cosh), _np(np.sinh)),
    "asinh": (_np(np.arcsinh), lambda x: 1.0 / _sqrt(x * x + 1.0)),
    "acosh": (_np(np.arccosh), lambda x: 1.0 / _sqrt(x * x - 1.0)),
    "atanh": (_np(np.arctanh), lambda x: 1.0 / (1.0 - x * x)),
    "sec": (lambda x: 1.0 / _cos(x), lambda x: _tan(x) / _cos(x)),
    "csc": (lambda x: 1.0 / _sin(x), lambda x: -1.0 / (_sin(x) * _tan(x))),
    "cot": (lambda x: 1.0 / _tan(x), lambda x: -(1.0 + 1.0 / _tan(x) ** 2)),
    "erf": (_erf, lambda x: 2.0 / math.sqrt(_PI) * _exp(-x * x)),
    "erfc": (_erfc, lambda x: -2.0 / math.sqrt(_PI) * _exp(-x * x)),
    "ncdf": (lambda x: 0.5 * _erfc(-x / math.sqrt(2.0)), lambda x: _exp(-0.5 * x * x) / math.sqrt(2.0 * _PI)),
    "sinc": (lambda x: _sinc(x)[0], lambda x: _sinc(x)[1]),
    "not": (lambda x: 0.0 if x != 0 else 1.0, lambda x: 0.0),
    "sgn": (lambda x: 1.0 if x > 0 else (-1.0 if x < 0 else 0.0), lambda x: 0.0),
    "floor": (_floor, lambda x: 0.0), "ceil": (_ceil, lambda x: 0.0), "round": (_round, lambda x: 0.0),
    "trunc": (_trunc, lambda x: 0.0), "frac": (lambda x: x - _trunc(x), lambda x: 1.0),
    "deg2rad": (lambda x: x * (_PI / 180.0), lambda x: _PI / 180.0),
    "rad2deg": (lambda x: x * (180.0 / _PI), lambda x: 180.0 / _PI),
    "deg2grad": (lambda x: x * (10.0 / 9.0), lambda x: 10.0 / 9.0),
    "grad2deg": (lambda x: x * (9.0 / 10.0), lambda x: 9.0 / 10.0),
}

_FUNC_NAMES = set(_FUNCS1) | {"min", "max", "sum", "avg", "mul", "mand", "mor", "pow", "atan2", "mod", "hypot",
                               "logn", "root", "roundn", "equal", "not_equal", "shl", "shr", "if", "clamp",
                               "iclamp", "inrange"}
_RESERVED = {"assert", "break", "case", "continue", "const", "default", "false", "for", "if", "else", "ilike",
             "in", "like", "and", "nand", "nor", "not", "null", "or", "repeat", "return", "shl", "shr", "swap",
             "switch", "true", "until", "var", "while", "xnor", "xor"}
# binary operators: token -> (left precedence, right precedence, name)
_BIN = {"+": (7, 8, "add"), "-": (7, 8, "sub"), "*": (10, 11, "mul"), "/": (10, 11, "div"),
        "%": (10, 11, "mod"), "^": (12, 12, "pow"), "<": (5, 6, "lt"), "<=": (5, 6, "le"), ">": (5, 6, "gt"),
        ">=": (5, 6, "ge"), "==": (5, 6, "eq"), "=": (5, 6, "eq"), "!=": (5, 6, "ne"), "<>": (5, 6, "ne"),
        "and": (3, 4, "and"), "nand": (3, 4, "nand"), "or": (1, 2, "or"), "nor": (1, 2, "nor"),
        "xor": (1, 2, "xor"), "xnor": (1, 2, "xnor")}


def _binary(name, a, b):
    """Value and partials (da, db) of a binary operation."""
    x, y = a.v, b.v
    t = lambda c: 1.0 if c else 0.0
    if name == "add":
        return x + y, 1.0, 1.0
    if name == "sub":
        return x - y, 1.0, -1.0
    if name == "mul":
        return x * y, y, x
    if name == "div":
        with np.errstate(all="ignore"):
            return float(np.float64(x) / y), float(1.0 / np.float64(y)), float(-np.float64(x) / (np.float64(y) * y))
    if name == "pow":
        v = _pow(x, y)
        return v, y * _pow(x, y - 1.0), (v * _log(x) if x > 0 else 0.0)
    if name == "mod":
        return _fmod(x, y), 1.0, -_trunc(x / y)
    if name in ("lt", "le", "gt", "ge", "eq", "ne"):
        r = {"lt": x < y, "le": x <= y, "gt": x > y, "ge": x >= y, "eq": x == y, "ne": x != y}[name]
        return t(r), 0.0, 0.0
    p, q = x != 0, y != 0
    r = {"and": p and q, "nand": not (p and q), "or": p or q, "nor": not (p or q), "xor": p != q,
         "xnor": p == q}[name]
    return t(r), 0.0, 0.0


def _lex(expr):
    toks, i = [], 0
    while i < len(expr):
        ch = expr[i]
        if ch.isspace():
            i += 1
        elif ch.isdigit() or (ch == "." and i + 1 < len(expr) and expr[i + 1].isdigit()):
            j = i
            while j < len(expr) and expr[j].isdigit():
                j += 1
            if j < len(expr) and expr[j] == ".":
                j += 1
                while j < len(expr) and expr[j].isdigit():
                    j += 1
            if j < len(expr) and expr[j] in "eE":
                k = j + 1
                if k < len(expr) and expr[k] in "+-":
                    k += 1
                if k < len(expr) and expr[k].isdigit():
                    while k < len(expr) and expr[k].isdigit():
                        k += 1
                    j = k
            toks.append(("num", float(expr[i:j])))
            i = j
        elif ch.isalpha() or ch == "_":
            j = i + 1
            while j < len(expr) and (expr[j].isalnum() or expr[j] in "_."):
                j += 1
            toks.append(("id", expr[i:j]))
            i = j
        elif ch in "&|":
            toks.append(("id", "and" if ch == "&" else "or"))
            i += 1
        elif expr[i:i + 2] in ("<=", ">=", "==", "!=", "<>"):
            toks.append(("op", expr[i:i + 2]))
            i += 2
        elif ch in "+-*/%^<>=()[]{},?:":
            toks.append(("op", ch))
            i += 1
        else:
            raise ValueError("unexpected character %r" % ch)
    plain = lambda t: t[0] == "id" and t[1].lower() not in _RESERVED
    out = []
    for k, t in enumerate(toks):   # implicit multiplication, as exprtk inserts it
        if k:
            a = toks[k - 1]
            if ((a[0] == "num" and (plain(t) or t in (("op", "("), ("op", "["), ("op", "{")))) or
                    (plain(a) and (t[0] == "num" or plain(t))) or
                    (plain(a) and a[1].lower() not in _FUNC_NAMES and t in (("op", "("), ("op", "["), ("op", "{"))) or
                    (a in (("op", ")"), ("op", "]"), ("op", "}")) and (t[0] == "num" or plain(t)))):
                out.append(("op", "*"))
        out.append(t)
    return out


def eval_expr(expr, values):
    """Evaluate a DIM expression over symbol values -> (value, {sym: d/dsym}).

    An independent restatement of the expression language exprtk::parser<double>
    accepts with default settings (src/grids/DimSet.cu:54-66): precedence
    (low -> high) ternary ?:, or/nor/xor/xnor, and/nand, comparisons, + -,
    * / %, unary minus, ^ (right-associative); functions, if(c,a,b) and the
    variadic min/max/sum/avg/mul/mand/mor; implicit multiplication; names
    case-insensitive.  Derivatives are exact (forward mode) where exprtk takes
    a five-point difference."""
    syms = list(values.keys())
    low = {s.lower(): s for s in reversed(syms)}
    nd = len(syms)
    toks = _lex(expr) + [("end", None)]
    pos = [0]

    def peek():
        return toks[pos[0]]

    def take():
        t = toks[pos[0]]
        pos[0] += 1
        return t

    def const(v):
        return _Dual(v, [0.0] * nd)

    def comb(v, parts):   # value v with partials (coefficient, operand) pairs; zero partials ignored
        d = [0.0] * nd
        for c, a in parts:
            if c != 0.0:
                d = [x + c * y for x, y in zip(d, a.d)]
        return _Dual(v, d)

    def close(open_):
        want = {"(": ")", "[": "]", "{": "}"}[open_]
        if take() != ("op", want):
            raise ValueError("expected %r" % want)

    def call(name, args):
        n = len(args)
        if name in _FUNCS1:
            assert n == 1, name
            f, df = _FUNCS1[name]
            a = args[0]
            return comb(f(a.v), [(df(a.v), a)])
        if name in ("min", "max", "sum", "avg", "mul", "mand", "mor"):
            acc = args[0]
            if n == 1 and name in ("mand", "mor"):
                return const(1.0 if acc.v != 0 else 0.0)
            for b in args[1:]:
                if name == "min":
                    acc = b if b.v < acc.v else acc
                elif name == "max":
                    acc = b if acc.v < b.v else acc
                elif name in ("sum", "avg"):
                    acc = comb(acc.v + b.v, [(1.0, acc), (1.0, b)])
                elif name == "mul":
                    acc = comb(acc.v * b.v, [(b.v, acc), (acc.v, b)])
                else:
                    acc = const(_binary("and" if name == "mand" else "or", acc, b)[0])
            if name == "avg":
                acc = comb(acc.v / n, [(1.0 / n, acc)])
            return acc
        if name in ("pow", "atan2", "mod", "hypot", "logn", "root", "roundn", "equal", "not_equal", "shl", "shr"):
            assert n == 2, name
            a, b = args
            x, y = a.v, b.v
            if name == "pow":
                v, da, db = _binary("pow", a, b)
            elif name == "mod":
                v, da, db = _binary("mod", a, b)
            elif name == "atan2":
                r2 = x * x + y * y
                v, da, db = math.atan2(x, y), y / r2, -x / r2
            elif name == "hypot":
                v = _sqrt(x * x + y * y)
                v, da, db = v, x / v, y / v
            elif name == "logn":
                v = _log(x) / _log(y)
                v, da, db = v, 1.0 / (x * _log(y)), -v / (y * _log(y))
            elif name == "root":
                v, da, db = _root(x, y)
            elif name == "roundn":
                p = 10.0 ** max(0, min(16, int(math.floor(y))))
                v, da, db = (_ceil(x * p - 0.5) if x < 0 else _floor(x * p + 0.5)) / p, 0.0, 0.0
            elif name in ("equal", "not_equal"):
                e = _near(x, y)
                v, da, db = (1.0 if e == (name == "equal") else 0.0), 0.0, 0.0
            else:
                s = 2.0 ** int(y)
                s = s if name == "shl" else 1.0 / s
                v, da, db = x * s, s, 0.0
            return comb(v, [(da, a), (db, b)])
        if name in ("if", "clamp", "iclamp", "inrange"):
            assert n == 3, name
            a, b, c = args
            if name == "if":
                return b if a.v != 0 else c
            if name == "clamp":
                return a if b.v < a.v else (c if b.v > c.v else b)
            if name == "iclamp":
                if b.v <= a.v or b.v >= c.v:
                    return b
                return a if 2.0 * b.v <= c.v + a.v else c
            return const(0.0 if (b.v < a.v or b.v > c.v) else 1.0)
        raise ValueError("unknown function " + name)

    def branch():
        t = take()
        if t == ("op", "-"):
            v = expression(11)
            return _Dual(-v.v, [-x for x in v.d])
        if t == ("op", "+"):
            return expression(13)
        if t[0] == "num":
            return const(t[1])
        if t in (("op", "("), ("op", "["), ("op", "{")):
            v = expression(0)
            close(t[1])
            return v
        if t[0] == "id":
            name, lname = t[1], t[1].lower()
            nxt = peek()
            if nxt in (("op", "("), ("op", "["), ("op", "{")) and lname in _FUNC_NAMES:
                take()
                args = [expression(0)]
                while peek() == ("op", ","):
                    take()
                    args.append(expression(0))
                close(nxt[1])
                return call(lname, args)
            sym = name if name in values else low.get(lname)
            if sym is not None:
                d = [0.0] * nd
                d[syms.index(sym)] = 1.0
                return _Dual(values[sym], d)
            consts = {"true": 1.0, "false": 0.0, "pi": math.pi, "e": math.e}
            if lname in consts:
                return const(consts[lname])
            raise ValueError("unknown symbol " + name)
        raise ValueError("bad token %r" % (t,))

    def expression(prec):
        v = branch()
        while True:
            t = peek()
            key = t[1] if t[0] == "op" else (t[1].lower() if t[0] == "id" else None)
            op = _BIN.get(key) if t[0] in ("op", "id") else None
            if op is None or op[0] < prec:
                break
            take()
            r = expression(op[1])
            val, da, db = _binary(op[2], v, r)
            v = comb(val, [(da, v), (db, r)])
        if prec == 0 and peek() == ("op", "?"):
            take()
            a = expression(0)
            if take() != ("op", ":"):
                raise ValueError("expected ':'")
            b = expression(0)
            v = a if v.v != 0 else b
        return v

    res = expression(0)
    if peek()[0] != "end":
        raise ValueError("trailing tokens in expression")
    return res.v, dict(zip(syms, res.d))
