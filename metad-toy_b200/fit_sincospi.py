"""Regenerates the coefficients of sin(pi f) = f P(f^2) and cos(pi f) = Q(f^2)
used by halfturn_sincos_f32 (csrc/common.cuh): near-minimax polynomials on
f in [0, 1/2] by Lawson's algorithm (least squares on Chebyshev and uniform
nodes, the weights raised where the error peaks, 30 rounds), P of degree 4
and Q of degree 5 in f^2.  Prints the coefficients and the maximum absolute
errors in FP64 arithmetic.

    python metad-toy_b200/fit_sincospi.py
"""
import math

import numpy as np


def lawson(f, nterms, x, rounds=30):
    A = np.stack([x ** (2 * k) for k in range(nterms)], 1)
    y = f(x)
    w = np.ones_like(x)
    for _ in range(rounds):
        c, *_ = np.linalg.lstsq(A * w[:, None], y * w, rcond=None)
        e = np.abs(A @ c - y)
        w = w * (1.0 + (e / e.max()) ** 2)
    return c


def main():
    x = np.concatenate([np.cos(np.linspace(0.0, math.pi, 20001)) * 0.25 + 0.25, np.linspace(0.0, 0.5, 20001)])
    safe = np.where(x == 0.0, 1.0, x)
    p = lawson(lambda z: np.where(z == 0.0, math.pi, np.sin(math.pi * z) / safe), 5, x)
    q = lawson(lambda z: np.cos(math.pi * z), 6, x)
    sp = x * (np.stack([x ** (2 * k) for k in range(5)], 1) @ p)
    cq = np.stack([x ** (2 * k) for k in range(6)], 1) @ q
    print("P", [repr(float(v)) for v in p], "max error", float(np.abs(sp - np.sin(math.pi * x)).max()))
    print("Q", [repr(float(v)) for v in q], "max error", float(np.abs(cq - np.cos(math.pi * x)).max()))


if __name__ == "__main__":
    main()
