"""The S(k) kernels' sin(pi f) / cos(pi f) polynomials (csrc/common.cuh,
halfturn_sincos_f32): the constants in the source are the ones
fit_sincospi.py produces, their error in exact arithmetic is below the
stated bounds, and an FP32 emulation of the device evaluation (the same
FMA sequence, the half-turn reduction and the sign flip) stays within 2e-7
of sin and cos over phases of a few hundred half turns."""
import math
import os
import re
import runpy

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "metad-toy_b200", "csrc", "common.cuh")


def _source_constants():
    text = open(SRC).read()
    vals = {}
    for name, v in re.findall(r"(kSinP\d|kCosQ\d) = \(float\)(-?[0-9.e-]+)", text):
        vals[name] = float(v)
    p = [vals["kSinP%d" % k] for k in range(5)]
    q = [vals["kCosQ%d" % k] for k in range(6)]
    return p, q


def test_source_constants_are_the_fit(capsys):
    runpy.run_path(os.path.join(ROOT, "metad-toy_b200", "fit_sincospi.py"), run_name="__main__")
    out = capsys.readouterr().out
    fit_p = [float(v.strip("'")) for v in re.search(r"P \[(.*?)\]", out).group(1).split(", ")]
    fit_q = [float(v.strip("'")) for v in re.search(r"Q \[(.*?)\]", out).group(1).split(", ")]
    p, q = _source_constants()
    assert p == fit_p and q == fit_q


def test_polynomial_error_bounds():
    p, q = _source_constants()
    z = np.linspace(0.0, 0.5, 200001)
    s = z * np.polyval(p[::-1], z * z)
    c = np.polyval(q[::-1], z * z)
    assert np.abs(s - np.sin(math.pi * z)).max() < 7e-9
    assert np.abs(c - np.cos(math.pi * z)).max() < 3e-10


def test_fp32_device_evaluation_emulated():
    P, Q = (np.array(v, dtype=np.float32) for v in _source_constants())

    def fma(a, b, c):   # the product and sum in FP64, then one rounding to FP32
        return (a.astype(np.float64) * np.float64(b) + c.astype(np.float64)).astype(np.float32)

    u = np.random.default_rng(3).uniform(-400.0, 400.0, 1_000_000)
    t = u + 6755399441055744.0
    n = t - 6755399441055744.0
    f = (u - n).astype(np.float32)
    z2 = (f * f).astype(np.float32)
    ps = fma(z2, P[4], np.full_like(z2, P[3]))
    for k in (2, 1, 0):
        ps = fma(ps, z2, np.full_like(z2, P[k]))
    s0 = (ps * f).astype(np.float32)
    qc = fma(z2, Q[5], np.full_like(z2, Q[4]))
    for k in (3, 2, 1, 0):
        qc = fma(qc, z2, np.full_like(z2, Q[k]))
    sign = np.where(np.mod(n, 2) == 0, 1.0, -1.0)
    assert np.abs(sign * s0 - np.sin(math.pi * u)).max() < 2e-7
    assert np.abs(sign * qc - np.cos(math.pi * u)).max() < 2e-7
