// expr_ops.h -- the operations of the DIM expression bytecode: arity, value
// and partial derivatives, shared by the host evaluator (expr.cpp) and the
// device evaluator of the bias kernels (bias.cu).
//
// Semantics follow exprtk as the reference uses it (src/grids/DimSet.cu:54-97
// compiles every DIM with exprtk::parser<double> and default settings):
// comparisons and logic give 1 or 0 (a value is true when it is not 0),
// `if(c, a, b)` and `c ? a : b` select a branch, min/max keep the first of
// equal arguments, round is half away from zero (floor(v + 0.5) / ceil(v - 0.5)),
// roundn(x, n) rounds to n decimals (n clamped to [0, 16]), root(x, n) of a
// negative x is defined for odd integer n, equal() compares within a relative
// 1e-10, shl/shr scale by a power of two.  Derivatives are exact: 0 on the
// flat pieces of comparisons, logic, floor/ceil/round/trunc/sgn, the chosen
// branch of a selection, the chosen argument of min/max/clamp.
#pragma once

#include <math.h>

#ifdef __CUDACC__
#define MTD_EXPR_HD __host__ __device__ __forceinline__
#else
#define MTD_EXPR_HD inline
#endif

namespace mtd {

enum ExprOp {
    // leaves
    EOP_CONST = 0, EOP_SYM,
    // binary
    EOP_ADD, EOP_SUB, EOP_MUL, EOP_DIV, EOP_POW,
    // unary
    EOP_NEG, EOP_SIN, EOP_COS, EOP_TAN, EOP_ASIN, EOP_ACOS, EOP_ATAN, EOP_EXP, EOP_LOG, EOP_LOG10,
    EOP_SQRT, EOP_ABS, EOP_TANH, EOP_SINH, EOP_COSH,
    // binary
    EOP_MIN, EOP_MAX, EOP_ATAN2,
    EOP_MOD, EOP_LT, EOP_LE, EOP_GT, EOP_GE, EOP_EQ, EOP_NE, EOP_AND, EOP_OR, EOP_XOR, EOP_NAND, EOP_NOR,
    EOP_XNOR, EOP_HYPOT, EOP_LOGN, EOP_ROOT, EOP_ROUNDN, EOP_EQUAL, EOP_NEQUAL, EOP_SHL, EOP_SHR,
    // unary
    EOP_NOT, EOP_SGN, EOP_FLOOR, EOP_CEIL, EOP_ROUND, EOP_TRUNC, EOP_FRAC, EOP_SEC, EOP_CSC, EOP_COT,
    EOP_ASINH, EOP_ACOSH, EOP_ATANH, EOP_LOG2, EOP_LOG1P, EOP_EXPM1, EOP_ERF, EOP_ERFC, EOP_NCDF, EOP_SINC,
    EOP_DEG2RAD, EOP_RAD2DEG, EOP_DEG2GRAD, EOP_GRAD2DEG,
    // ternary: select (if / ?:), clamp, iclamp, inrange
    EOP_SEL, EOP_CLAMP, EOP_ICLAMP, EOP_INRANGE,
    EOP_COUNT
};

MTD_EXPR_HD int expr_arity(int op) {
    if (op == EOP_CONST || op == EOP_SYM) return 0;
    if ((op >= EOP_ADD && op <= EOP_POW) || (op >= EOP_MIN && op <= EOP_SHR)) return 2;
    if (op >= EOP_SEL && op <= EOP_INRANGE) return 3;
    return 1;
}

MTD_EXPR_HD double expr_truth(double v) { return v != 0.0 ? 1.0 : 0.0; }

// Exact powers of ten for roundn.
MTD_EXPR_HD double expr_pow10(int k) {
    double p = 1.0;
    for (int i = 0; i < k; ++i) p *= 10.0;
    return p;
}

// exprtk's round: half away from zero through floor / ceil.
MTD_EXPR_HD double expr_round(double v) { return v < 0.0 ? ceil(v - 0.5) : floor(v + 0.5); }

// One operation on its operands a[0 .. arity-1]: returns the value and writes
// d[k] = d value / d a[k].
MTD_EXPR_HD double expr_apply(int op, const double *a, double *d) {
    const double kPiE = 3.14159265358979323846;
    d[0] = d[1] = d[2] = 0.0;
    const double x = a[0];
    const double y = a[1];
    double v = 0.0;
    switch (op) {
    case EOP_ADD: v = x + y; d[0] = 1.0; d[1] = 1.0; break;
    case EOP_SUB: v = x - y; d[0] = 1.0; d[1] = -1.0; break;
    case EOP_MUL: v = x * y; d[0] = y; d[1] = x; break;
    case EOP_DIV: v = x / y; d[0] = 1.0 / y; d[1] = -x / (y * y); break;
    case EOP_POW:
        v = pow(x, y);
        d[0] = y * pow(x, y - 1.0);
        d[1] = x > 0.0 ? v * log(x) : 0.0;
        break;
    case EOP_MIN: if (y < x) { v = y; d[1] = 1.0; } else { v = x; d[0] = 1.0; } break;
    case EOP_MAX: if (x < y) { v = y; d[1] = 1.0; } else { v = x; d[0] = 1.0; } break;
    case EOP_ATAN2: {
        const double r2 = x * x + y * y;
        v = atan2(x, y);
        d[0] = y / r2;
        d[1] = -x / r2;
        break;
    }
    case EOP_MOD: v = fmod(x, y); d[0] = 1.0; d[1] = -trunc(x / y); break;
    case EOP_LT: v = x < y ? 1.0 : 0.0; break;
    case EOP_LE: v = x <= y ? 1.0 : 0.0; break;
    case EOP_GT: v = x > y ? 1.0 : 0.0; break;
    case EOP_GE: v = x >= y ? 1.0 : 0.0; break;
    case EOP_EQ: v = x == y ? 1.0 : 0.0; break;
    case EOP_NE: v = x != y ? 1.0 : 0.0; break;
    case EOP_AND: v = (x != 0.0 && y != 0.0) ? 1.0 : 0.0; break;
    case EOP_OR: v = (x != 0.0 || y != 0.0) ? 1.0 : 0.0; break;
    case EOP_XOR: v = expr_truth(x) != expr_truth(y) ? 1.0 : 0.0; break;
    case EOP_NAND: v = (x != 0.0 && y != 0.0) ? 0.0 : 1.0; break;
    case EOP_NOR: v = (x != 0.0 || y != 0.0) ? 0.0 : 1.0; break;
    case EOP_XNOR: v = expr_truth(x) == expr_truth(y) ? 1.0 : 0.0; break;
    case EOP_HYPOT: v = sqrt(x * x + y * y); d[0] = x / v; d[1] = y / v; break;
    case EOP_LOGN: {
        const double lb = log(y);
        v = log(x) / lb;
        d[0] = 1.0 / (x * lb);
        d[1] = -v / (y * lb);
        break;
    }
    case EOP_ROOT:
        if (x < 0.0) {
            const bool odd = (y == trunc(y)) && (fmod(y, 2.0) != 0.0);
            v = odd ? -pow(-x, 1.0 / y) : NAN;
        } else {
            v = pow(x, 1.0 / y);
        }
        d[0] = v / (y * x);
        d[1] = x != 0.0 ? -v * log(fabs(x)) / (y * y) : 0.0;
        break;
    case EOP_ROUNDN: {
        int k = (int)floor(y);
        k = k < 0 ? 0 : (k > 16 ? 16 : k);
        const double p = expr_pow10(k);
        v = (x < 0.0 ? ceil(x * p - 0.5) : floor(x * p + 0.5)) / p;
        break;
    }
    case EOP_EQUAL: {
        const double ax = fabs(x), ay = fabs(y);
        const double m = ax > ay ? ax : ay;
        v = fabs(x - y) <= (m > 1.0 ? m : 1.0) * 1e-10 ? 1.0 : 0.0;
        break;
    }
    case EOP_NEQUAL: {
        const double ax = fabs(x), ay = fabs(y);
        const double m = ax > ay ? ax : ay;
        v = fabs(x - y) > (m > 1.0 ? m : 1.0) * 1e-10 ? 1.0 : 0.0;
        break;
    }
    case EOP_SHL: { const double s = pow(2.0, (double)(int)y); v = x * s; d[0] = s; break; }
    case EOP_SHR: { const double s = 1.0 / pow(2.0, (double)(int)y); v = x * s; d[0] = s; break; }
    case EOP_NEG: v = -x; d[0] = -1.0; break;
    case EOP_SIN: v = sin(x); d[0] = cos(x); break;
    case EOP_COS: v = cos(x); d[0] = -sin(x); break;
    case EOP_TAN: v = tan(x); d[0] = 1.0 + v * v; break;
    case EOP_ASIN: v = asin(x); d[0] = 1.0 / sqrt(1.0 - x * x); break;
    case EOP_ACOS: v = acos(x); d[0] = -1.0 / sqrt(1.0 - x * x); break;
    case EOP_ATAN: v = atan(x); d[0] = 1.0 / (1.0 + x * x); break;
    case EOP_EXP: v = exp(x); d[0] = v; break;
    case EOP_LOG: v = log(x); d[0] = 1.0 / x; break;
    case EOP_LOG10: v = log10(x); d[0] = 1.0 / (x * 2.30258509299404568402); break;
    case EOP_SQRT: v = sqrt(x); d[0] = 0.5 / v; break;
    case EOP_ABS: v = fabs(x); d[0] = (x > 0.0) - (x < 0.0); break;
    case EOP_TANH: v = tanh(x); d[0] = 1.0 - v * v; break;
    case EOP_SINH: v = sinh(x); d[0] = cosh(x); break;
    case EOP_COSH: v = cosh(x); d[0] = sinh(x); break;
    case EOP_NOT: v = x != 0.0 ? 0.0 : 1.0; break;
    case EOP_SGN: v = x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); break;
    case EOP_FLOOR: v = floor(x); break;
    case EOP_CEIL: v = ceil(x); break;
    case EOP_ROUND: v = expr_round(x); break;
    case EOP_TRUNC: v = trunc(x); break;
    case EOP_FRAC: v = x - trunc(x); d[0] = 1.0; break;
    case EOP_SEC: v = 1.0 / cos(x); d[0] = v * tan(x); break;
    case EOP_CSC: v = 1.0 / sin(x); d[0] = -v / tan(x); break;
    case EOP_COT: v = 1.0 / tan(x); d[0] = -(1.0 + v * v); break;
    case EOP_ASINH: v = asinh(x); d[0] = 1.0 / sqrt(x * x + 1.0); break;
    case EOP_ACOSH: v = acosh(x); d[0] = 1.0 / sqrt(x * x - 1.0); break;
    case EOP_ATANH: v = atanh(x); d[0] = 1.0 / (1.0 - x * x); break;
    case EOP_LOG2: v = log2(x); d[0] = 1.0 / (x * 0.69314718055994530942); break;
    case EOP_LOG1P: v = log1p(x); d[0] = 1.0 / (1.0 + x); break;
    case EOP_EXPM1: v = expm1(x); d[0] = exp(x); break;
    case EOP_ERF: v = erf(x); d[0] = 1.12837916709551257390 * exp(-x * x); break;
    case EOP_ERFC: v = erfc(x); d[0] = -1.12837916709551257390 * exp(-x * x); break;
    case EOP_NCDF:   // 0.5 erfc(-x / sqrt 2); derivative the normal density
        v = 0.5 * erfc(-x / 1.41421356237309504880);
        d[0] = 0.39894228040143267794 * exp(-0.5 * x * x);
        break;
    case EOP_SINC:   // sin(x) / x, 1 within one double epsilon of 0
        if (fabs(x) >= 2.220446049250313e-16) {
            v = sin(x) / x;
            d[0] = (cos(x) - v) / x;
        } else {
            v = 1.0;
        }
        break;
    case EOP_DEG2RAD: v = x * (kPiE / 180.0); d[0] = kPiE / 180.0; break;
    case EOP_RAD2DEG: v = x * (180.0 / kPiE); d[0] = 180.0 / kPiE; break;
    case EOP_DEG2GRAD: v = x * (10.0 / 9.0); d[0] = 10.0 / 9.0; break;
    case EOP_GRAD2DEG: v = x * (9.0 / 10.0); d[0] = 9.0 / 10.0; break;
    case EOP_SEL: if (x != 0.0) { v = y; d[1] = 1.0; } else { v = a[2]; d[2] = 1.0; } break;
    case EOP_CLAMP:   // clamp(lo, v, hi)
        if (y < x) { v = x; d[0] = 1.0; }
        else if (y > a[2]) { v = a[2]; d[2] = 1.0; }
        else { v = y; d[1] = 1.0; }
        break;
    case EOP_ICLAMP:   // iclamp(lo, v, hi): v outside (lo, hi), else the nearer end
        if (y <= x || y >= a[2]) { v = y; d[1] = 1.0; }
        else if (2.0 * y <= a[2] + x) { v = x; d[0] = 1.0; }
        else { v = a[2]; d[2] = 1.0; }
        break;
    case EOP_INRANGE: v = (y < x) ? 0.0 : ((y > a[2]) ? 0.0 : 1.0); break;
    default: v = NAN; break;
    }
    return v;
}

}  // namespace mtd
