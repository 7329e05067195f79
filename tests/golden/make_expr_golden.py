"""Generates tests/golden/expr_exprtk.json: DIM expressions evaluated by exprtk
itself, the way the reference evaluates them (src/grids/DimSet.cu:54-97:
parser<double> with default settings, one variable per symbol, no
add_constants(), value() and exprtk::derivative per symbol).

Run in a container that has the reference checkout, after
`make -C oracle ref REF_DIR=<checkout>` (builds oracle/_ref/libexprref.so from
the checkout's third_party/exprtk.hpp and oracle/expr_harness.cpp):

    python tests/golden/make_expr_golden.py

Each record: the expression, the symbol values, and either exprtk's value and
derivatives or "error": true when exprtk rejects the expression.  The points
sit away from every discontinuity by far more than exprtk's difference step
(2e-8), so its derivatives are those of the smooth piece.
"""
import ctypes as C
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

# (expression, list of symbol-value dicts)
P2 = [{"v1": 0.3, "v2": 0.7}, {"v1": -1.25, "v2": 2.5}, {"v1": 0.8, "v2": -0.45}]
PP = [{"v1": 0.3, "v2": 0.7}, {"v1": 1.75, "v2": 0.45}]        # positive arguments
P3 = [{"v1": 0.3, "v2": 0.7, "v3": -0.2}, {"v1": -0.6, "v2": 0.1, "v3": 0.9}]
CASES = [
    # arithmetic and precedence
    ("v1", P2), ("v1+v2", P2), ("(v1+v2)/2", P2), ("v1*v2", P2), ("v1-v2-0.25", P2),
    ("v1/v2/3", P2), ("2^3^0.5 + v1", P2), ("-v1^2", P2), ("-2^2*v1", P2), ("v1^-2", P2),
    ("v1 % 0.35 + v2", P2), ("3 % v2", PP), ("-v1*v2 + +v2", P2), ("v1^2^0.5", PP),
    ("1.5e-1*v1 + .5 - 2E1*v2", P2),
    # comparisons and logic
    ("v1 < v2", P2), ("v1 <= v2", P2), ("v1 > v2", P2), ("v1 >= v2", P2), ("v1 == v2", P2),
    ("v1 = v1", P2), ("v1 != v2", P2), ("v1 <> v2", P2), ("(v1 < v2) + 2*(v1 > 0)", P2),
    ("v1 < v2 and v2 > 0", P2), ("v1 > v2 or v2 > 0", P2), ("v1 > 0 xor v2 > 0", P2),
    ("v1 > 0 nand v2 > 0", P2), ("v1 > 0 nor v2 > 5", P2), ("v1 > 0 xnor v2 > 0", P2),
    ("v1 > 0 & v2 > 0", P2), ("v1 > 5 | v2 > 0", P2), ("not(v1 > v2)", P2),
    ("v1 + v2 > 0.5 and v1 < 1 or v2 < -1", P2), ("true + false*v1 + v2", P2),
    # selection
    ("v1 > v2 ? v1*v1 : 2*v2", P2), ("v1 < 0 ? -v1 : v1 > 0.5 ? v1 : v2", P2),
    ("if(v1 > 0, v1*v2, v2 - v1)", P2), ("v1 + (v2 > 0 ? v2 : 0)", P2),
    ("clamp(0, v1*2, 1)", P2), ("clamp(-1, v1 + v2, 0.9)", P2), ("iclamp(0, v1, 1)", P2),
    ("iclamp(0, v2, 1) + iclamp(-2, v1, 1)", P2), ("inrange(0, v1, 1) + v2", P2),
    # variadic
    ("min(v1, v2)", P2), ("max(v1, v2)", P2), ("min(v1, v2, 0.1)", P2), ("max(v1, v2, v1*v2, -3)", P2),
    ("sum(v1, v2, 1)", P2), ("avg(v1, v2)", P2), ("avg(v1, v2, 2*v1)", P2), ("mul(v1, v2, 3)", P2),
    ("mand(v1 > 0, v2 > 0, 1)", P2), ("mor(v1 > 1, v2 > 1)", P2), ("min(v1)", P2),
    # functions of one argument
    ("sin(v1) + cos(v2)", P2), ("tan(v1*v2)", P2), ("asin(v1/2) + acos(v2/3)", P2), ("atan(v1 - v2)", P2),
    ("exp(v1) - log(v2)", PP), ("log10(v1) + log2(v2)", PP), ("log1p(v1) + expm1(v2)", PP),
    ("sqrt(v1 + v2*v2)", PP), ("abs(v1 - v2)", P2), ("tanh(v1) + sinh(v2) - cosh(v1)", P2),
    ("sgn(v1) * v2", P2), ("floor(3*v1) + ceil(3*v2) + v1", P2), ("round(4.3*v1) + trunc(4.3*v2)", P2),
    ("frac(3.7*v1) + v2", P2), ("sec(v1) + csc(v2) + cot(v2)", P2), ("asinh(v1) + acosh(1.5 + v2*v2)", P2),
    ("atanh(v1/2)", P2), ("erf(v1) + erfc(v2)", P2), ("ncdf(v1 - v2)", P2), ("sinc(v1 + v2)", P2),
    ("deg2rad(10*v1) + rad2deg(v2)", P2), ("deg2grad(v1) + grad2deg(v2)", P2),
    # functions of two and three arguments
    ("pow(v1*v1 + 1, v2)", P2), ("atan2(v1, v2)", P2), ("mod(5*v1, 0.7) + v2", P2), ("hypot(v1, v2)", P2),
    ("logn(v1 + 2, 3) + logn(8, v2 + 2)", PP), ("root(v1 + 2, 3)", P2), ("root(-8*v1*v1 - 1, 3)", P2),
    ("roundn(v1*v2, 3) + v1", P2), ("roundn(3.14159*v1, 2.7)", P2), ("equal(v1, v1 + 1e-12)", P2),
    ("equal(v1, v2) + not_equal(v1, v2)", P2), ("shl(v1, 3) + shr(v2, 2)", P2),
    # implicit multiplication and case
    ("2v1 + 3v2", P2), ("2(v1 + v2)", P2), ("(v1 + 1)v2", P2), ("(v1 + 1)2", P2), ("v1 v2", P2),
    ("2sin(v1)", P2), ("SIN(V1) + Max(v1, V2)", P2),
    # three symbols
    ("v1*v2*v3 + v3^2", P3), ("v3 > 0 ? v1 : v2", P3), ("clamp(v3, v1, v2)", P3),
    # brackets
    ("[v1 + v2] * {v1 - v2}", P2),
    # a variable then a bracket multiplies; assignment (accepted by exprtk)
    ("v1(v2)", P2), ("v1 := 2", P2),
    # rejected by exprtk
    ("v1 +", P2), ("foo(v1)", P2), ("min()", P2), ("w9 + 1", P2), ("pi * v1", P2), ("e + v1", P2),
]


def main():
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libexprref.so"))
    lib.exref_eval.restype = C.c_int
    lib.exref_eval.argtypes = [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), C.POINTER(C.c_double),
                               C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_char_p, C.c_int]
    out = []
    for expr, points in CASES:
        for vals in points:
            names = list(vals)
            n = len(names)
            cn = (C.c_char_p * n)(*[s.encode() for s in names])
            cv = (C.c_double * n)(*[vals[s] for s in names])
            value = C.c_double()
            grad = (C.c_double * n)()
            err = C.create_string_buffer(512)
            rc = lib.exref_eval(expr.encode(), n, cn, cv, C.byref(value), grad, err, 512)
            rec = {"expr": expr, "values": vals}
            if rc:
                rec["error"] = True
            else:
                rec["value"] = value.value
                rec["grad"] = {s: grad[k] for k, s in enumerate(names)}
            out.append(rec)
    with open(os.path.join(HERE, "expr_exprtk.json"), "w") as f:
        json.dump(out, f, indent=0, allow_nan=True)
    print("wrote %d records" % len(out))


if __name__ == "__main__":
    main()
