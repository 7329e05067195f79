"""The oracle pinned against the reference's own arithmetic and known answers
(CPU only).

Pins:
  * Y_lm and dY_lm/dd at 256 bond vectors from the reference header itself
    (tests/golden/ylm_reference.npz, made by tests/golden/make_golden.py);
  * perfect-lattice Q4/Q6 of FCC (12 neighbours) and BCC (8 neighbours);
  * central finite differences of every CV gradient;
  * the reference's own HILLS file (format and content).
"""
import os

import numpy as np
import pytest

import oracle as O
import systems

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def test_ylm_matches_reference_header():
    z = np.load(os.path.join(GOLD, "ylm_reference.npz"))
    for l in (3, 4, 6):
        for i in range(z["d"].shape[0]):
            y = O.ylm(l, z["d"][i])
            ref = z["ylm%d" % l][i]
            assert np.max(np.abs(y.real - ref[0::2])) < 1e-13
            assert np.max(np.abs(y.imag - ref[1::2])) < 1e-13


def test_ylm_gradient_matches_reference_header():
    z = np.load(os.path.join(GOLD, "ylm_reference.npz"))
    for l in (4, 6):
        for i in range(z["d"].shape[0]):
            _, g = O.ylm_grad(l, z["d"][i])
            ref = z["dylm%d" % l][i].reshape(l + 1, 6)
            assert np.max(np.abs(g[:, 0].real - ref[:, 0])) < 1e-12
            assert np.max(np.abs(g[:, 0].imag - ref[:, 1])) < 1e-12
            assert np.max(np.abs(g[:, 1].real - ref[:, 2])) < 1e-12
            assert np.max(np.abs(g[:, 1].imag - ref[:, 3])) < 1e-12
            assert np.max(np.abs(g[:, 2].real - ref[:, 4])) < 1e-12
            assert np.max(np.abs(g[:, 2].imag - ref[:, 5])) < 1e-12


@pytest.mark.parametrize("l", [3, 4, 6])
def test_ylm_normalisation(l):
    rng = np.random.default_rng(l)
    for _ in range(20):
        y = O.ylm(l, rng.normal(size=3))
        s = abs(y[0]) ** 2 + 2 * np.sum(np.abs(y[1:]) ** 2)
        assert abs(s - (2 * l + 1) / (4 * np.pi)) < 1e-13


@pytest.mark.parametrize("lat,nc,a,rc,cap,q4,q6", [
    ("fcc", 4, 5.26, 3.9, 12, 0.190941, 0.574524),
    ("bcc", 4, 4.18, 3.7, 8, 0.509175, 0.628539),
])
def test_perfect_lattice_known_answers(lat, nc, a, rc, cap, q4, q6):
    x = systems.fcc(nc, a) if lat == "fcc" else systems.bcc(nc, a)
    L = [nc * a] * 3
    o4 = O.steinh_q(4, x, L, rc, cap, grad=False)
    o6 = O.steinh_q(6, x, L, rc, cap, grad=False)
    assert np.all(o4["nkept"] == cap)
    assert abs(o4["cv"] - q4) < 1e-6 and abs(o6["cv"] - q6) < 1e-6


def _fd(f, x, idx, h=1e-6):
    g = np.zeros((len(idx), 3))
    for a, i in enumerate(idx):
        for c in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, c] += h
            xm[i, c] -= h
            g[a, c] = (f(xp) - f(xm)) / (2 * h)
    return g


X0 = systems.jitter(systems.fcc(3, 5.26), 0.15, 7)
L0 = [3 * 5.26] * 3
IDX = [0, 5, 17, 40, 77]


@pytest.mark.parametrize("l", [4, 6])
@pytest.mark.parametrize("mode", ["AVE", "SW_FUNC"])
def test_steinh_q_gradient_fd(l, mode):
    sw = O.make_sw("FERMI", r0=0.4, alpha=10.0)
    o = O.steinh_q(l, X0, L0, 3.9, 18, mode=mode, swcv=sw)
    g = _fd(lambda x: O.steinh_q(l, x, L0, 3.9, 18, mode=mode, swcv=sw, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-7 * max(1.0, np.abs(g).max())


def test_steinh_q_binding_cap_gradient_fd():
    # rc 4.5 holds 12 neighbours, cap 10 binds; small steps keep the kept sets fixed
    o = O.steinh_q(6, X0, L0, 4.5, 10)
    g = _fd(lambda x: O.steinh_q(6, x, L0, 4.5, 10, grad=False)["cv"], X0, IDX, h=1e-7)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-6 * np.abs(g).max()


def test_reference_q_gradient_is_truncated():
    """The reference STEINH Q force omits terms (CV_Steinhardt_math.h:200-668);
    the oracle's exact gradient is the FD-consistent one."""
    z = np.load(os.path.join(GOLD, "q_grad_reference_faithful.npz"))
    for l in (4, 6):
        o = O.steinh_q(l, z["x"], z["L"], 3.9, 18)
        assert np.max(np.abs(o["grad"] - z["grad_exact%d" % l])) < 1e-14
        dev = np.max(np.abs(z["grad_ref%d" % l] - z["grad_exact%d" % l]))
        assert dev > 0.1 * np.abs(z["grad_exact%d" % l]).max()


@pytest.mark.parametrize("l", [4, 6])
@pytest.mark.parametrize("mode", ["MEAN_SOLID", "NSOLID", "FRAC"])
def test_steinh_l_gradient_fd(l, mode):
    swr = O.make_sw("FERMI", r0=3.9, alpha=-8.0)
    rl = O.sw_invert_for_eps(swr, 1e-6)
    swc = O.make_sw("FERMI", r0=0.3, alpha=20.0)
    o = O.steinh_l(l, X0, L0, rl, swr, 1e-6, swc, mode)
    g = _fd(lambda x: O.steinh_l(l, x, L0, rl, swr, 1e-6, swc, mode, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-7 * max(1.0, np.abs(g).max())


def test_steinh_l_step_switch_and_group_fd():
    grp = (np.arange(X0.shape[0]) % 3 != 0).astype(np.int32)
    sw = O.make_sw("STEP", r0=3.9)
    o = O.steinh_l(6, X0, L0, 3.9, sw, ingroup=grp)
    g = _fd(lambda x: O.steinh_l(6, x, L0, 3.9, sw, ingroup=grp, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-7


@pytest.mark.parametrize("mode", ["AVE", "COUNT"])
def test_debye_gradient_fd(mode):
    sw = O.make_sw("FERMI", r0=1.5, alpha=5.0)
    o = O.debye(X0, L0, 6.0, 2.8, mode=mode, sw=sw)
    g = _fd(lambda x: O.debye(x, L0, 6.0, 2.8, mode=mode, sw=sw, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-7 * max(1.0, np.abs(g).max())


def test_chemical_debye_gradient_fd_and_unit_weights():
    """STRU_FACTOR Chemical: pair terms times w(type_i) w(type_j); with all
    weights 1 it is the plain Debye CV exactly."""
    types = (np.arange(X0.shape[0]) % 3) + 1
    w = O.chem_type_weights(types, ctarget=2.0, sigma=0.8, cmap={3: 0.4})
    assert w[types == 3].max() == 0.4 and abs(w[types == 1][0] - np.exp(-1 / 1.28)) < 1e-15
    plain = O.debye(X0, L0, 6.0, 2.8)
    ones = O.debye(X0, L0, 6.0, 2.8, weights=np.ones(X0.shape[0]))
    assert ones["cv"] == plain["cv"] and np.array_equal(ones["grad"], plain["grad"])
    o = O.debye(X0, L0, 6.0, 2.8, weights=w)
    g = _fd(lambda x: O.debye(x, L0, 6.0, 2.8, weights=w, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-7 * max(1.0, np.abs(g).max())


@pytest.mark.parametrize("mode", ["AVE", "COUNT"])
def test_weight_chem_gradient_fd(mode):
    """WEIGHT_CHEM: P_i = 1 + sum_j w_i w_j s(r_ij) with the taper s alone as
    pair term (q_factor 0 in the shared Debye restatement)."""
    types = (np.arange(X0.shape[0]) % 2) + 1
    w = O.chem_type_weights(types, cmap={1: 0.1, 2: 3.0})
    sw = O.make_sw("FERMI", r0=12.0, alpha=2.0)
    o = O.debye(X0, L0, 3.0, 0.0, mode=mode, sw=sw, weights=w)
    g = _fd(lambda x: O.debye(x, L0, 3.0, 0.0, mode=mode, sw=sw, weights=w, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-7 * max(1.0, np.abs(g).max())


def test_sk_gradient_fd_and_bragg_peak():
    k = systems.kvectors(8, systems.KMAG_111, 5)
    o = O.sk(X0, k)
    g = _fd(lambda x: O.sk(x, k, grad=False)["cv"], X0, IDX)
    assert np.max(np.abs(g - o["grad"][IDX])) < 1e-6 * max(1.0, np.abs(g).max())
    # a perfect lattice at a <111> Bragg vector gives S = N
    x = systems.fcc(3, 5.26)
    kb = np.array([[1.0, 1.0, 1.0]]) * (2 * np.pi / 5.26)
    assert abs(O.sk(x, kb, grad=False)["Sk"][0] - x.shape[0]) < 1e-8


def test_switching_functions_restated():
    st = O.make_sw("STEP", r0=3.9)
    assert O.sw_f(st, 3.899) == 1.0 and O.sw_f(st, 3.9) == 0.0 and O.sw_df(st, 1.0) == 0.0
    fe = O.make_sw("FERMI", r0=1.0, alpha=20.0)
    assert abs(O.sw_f(fe, 1.0) - 0.5) < 1e-15
    ra = O.make_sw("RATIONAL", r0=1.25)
    x = 1.7
    assert abs(O.sw_f(ra, x) - 1 / (1 + (x / 1.25) ** 6)) < 1e-15
    for sw in (fe, ra, O.make_sw("TANH", r0=1.0, alpha=3.0), O.make_sw("RATIONAL", r0=1.0, n=5, m=9)):
        for x in (0.6, 0.95, 1.3):
            h = 1e-6
            fd = (O.sw_f(sw, x + h) - O.sw_f(sw, x - h)) / (2 * h)
            assert abs(fd - O.sw_df(sw, x)) < 1e-6
    # invert_for_eps (switch.h:339-367): the switch equals eps at the returned radius
    for sw in (O.make_sw("FERMI", r0=3.9, alpha=-8.0), O.make_sw("RATIONAL", r0=1.25), O.make_sw("TANH", r0=3.9, alpha=-4.0)):
        r = O.sw_invert_for_eps(sw, 1e-6)
        assert abs(O.sw_f(sw, r) - 1e-6) < 1e-9
    assert O.sw_invert_for_eps(O.make_sw("LINE"), 1e-6) == -1.0


def test_grid_deposit_and_interpolation():
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.02, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([0.4025, 0.6025])
    V, dV = g.value([0.4025, 0.6025])
    assert abs(V - 0.005) < 2e-4 and np.all(np.abs(dV) < 0.05)
    # interpolated values track the exact Gaussian away from the centre
    for p in ([0.43, 0.6], [0.4, 0.63], [0.37, 0.57]):
        Ve, dVe = O.hill_sum(np.array([[0.4025, 0.6025]]), np.array([0.005]), np.array([0.02]), np.array([p]))
        V, dV = g.value(p)
        assert abs(V - Ve[0]) < 2e-5
        assert np.max(np.abs(dV - dVe[0])) < 2e-3


def test_reference_hills_fixture_format():
    path = os.path.join(GOLD, "HILLS_1d_reference_fixture")
    lines = open(path).read().splitlines()
    assert lines[0] == "# step cv_values height sigma"
    rows = np.array([[float(t) for t in ln.split()] for ln in lines[1:] if ln.strip()])
    assert rows.shape == (238, 4)
    assert np.all(rows[:, 2] == 0.005) and np.all(rows[:, 3] == 0.01)
    assert rows[0, 0] == 555100 and rows[-1, 0] == 578800


def test_dim_expression_oracle():
    v, d = O.eval_expr("sqrt(v1^2+v2^2)*2 - exp(-v2)", {"v1": 0.3, "v2": 0.4})
    assert abs(v - (2 * 0.5 - np.exp(-0.4))) < 1e-15
    assert abs(d["v1"] - 1.2) < 1e-14 and abs(d["v2"] - (1.6 + np.exp(-0.4))) < 1e-14
