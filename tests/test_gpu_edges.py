"""Edge cases through the C ABI against the FP64 oracle: pairs sitting on the
cutoff to the last bit, two atoms in an open box (the reference's two-atom
toy deck), an empty group, zero atoms, a non-periodic dimension, a 3D
bias grid and a non-finite position.  Tolerances as in the parity tests: FP64 1e-9 relative on CVs and
bias, 1e-8 on forces; mixed 2e-5 and 2e-3 of the largest force component."""
import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-9, 1e-8), "mixed": (2e-5, 2e-3)}


def _simple_cubic(nc, a):
    g = np.arange(nc) * a
    x = np.stack(np.meshgrid(g, g, g, indexing="ij"), axis=-1).reshape(-1, 3)
    return np.ascontiguousarray(x), np.array([nc * a] * 3)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pairs_on_the_cutoff_decide_as_the_oracle(precision):
    """Simple cubic with a = cutoff: every nearest pair sits within an ulp of
    r = r_c, on either side depending on FP64 rounding of the coordinates;
    the neighbour sets (STEINH Q: r <= r_c; STEINH L STEP: r < r_0) must be
    the oracle's, which the CVs show (a flipped pair moves Q by ~1e-2)."""
    x, L = _simple_cubic(8, 3.9)
    args = ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "QG", "STEINH", "Q", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18,
            "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "QL", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "SYMBOL", "v1", "QG.AVE", "SYMBOL", "v2", "QL.MEAN_SOLID",
            "CV_dim", 2, "DIM", 1, 0, 1, 100, "v1", "DIM", 2, 0, 1, 100, "v2", "WT", 0]
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    oq = O.steinh_q(6, x, L, 3.9, 18)
    ol = O.steinh_l(6, x, L, 3.9, O.make_sw("STEP", r0=3.9), 1e-6, None, "MEAN_SOLID")
    tcv, _ = TOL[precision]
    cv = out[0][0]
    assert H.rel(cv[0], oq["cv"]) < tcv
    assert H.rel(cv[1], ol["cv"]) < tcv
    assert m.max_neighbors("QG") == oq["nrc"].max()
    assert m.max_neighbors("QL") == ol["nnb"].max()
    m.close()


def test_two_atoms_in_an_open_box():
    """Two atoms 3 A apart, no periodic dimension: one neighbour each, so
    Q6 = 1 and its gradient vanishes (the reference's two-atom toy)."""
    x = np.array([[20.0, 20.0, 20.0], [22.0, 21.0, 22.0]])
    L = np.array([50.0, 50.0, 50.0])
    m = mtd.Metad(H.fix_args_q(), precision="fp64")
    m.set_box([0, 0, 0], L, periodic=(0, 0, 0))
    f = np.zeros_like(x)
    m.post_force(0, x, f)
    o = O.steinh_q(6, x, L, 3.9, 18, periodic=(0, 0, 0))
    assert abs(m.cv[0] - 1.0) < 1e-12 and abs(o["cv"] - 1.0) < 1e-12
    assert np.abs(f).max() < 1e-12
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_non_periodic_dimension(precision):
    """A slab open in z (atoms near both z faces have no images)."""
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = systems.jitter(x, 0.05, 9)
    x[:, 2] = np.clip(x[:, 2], 1e-3, L[2] - 1e-3)
    args = H.fix_args_local()
    m = mtd.Metad(args, precision=precision)
    m.set_box([0, 0, 0], L, periodic=(1, 1, 0))
    f = np.zeros_like(x)
    m.post_force(0, np.ascontiguousarray(x), f)
    per = (1, 1, 0)
    sw = O.make_sw("STEP", r0=3.9)
    o4 = O.steinh_l(4, x, L, 3.9, sw, 1e-6, None, "MEAN_SOLID", periodic=per)
    o6 = O.steinh_l(6, x, L, 3.9, sw, 1e-6, None, "MEAN_SOLID", periodic=per)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    g.add_hill(s)
    V, dV = g.value(s)
    tcv, tf = TOL[precision]
    assert H.rel(m.cv, s) < tcv
    assert H.rel(m.compute_scalar(), V) < tcv
    assert H.rel(f, -(dV[0] * o4["grad"] + dV[1] * o6["grad"])) < tf
    m.close()


def test_empty_group_gives_zero_cv_and_no_force():
    """A CAL on a group no atom belongs to: N = 0, the AVE and MEAN_SOLID CVs
    are 0 (as the reference's guarded divisions give), forces untouched."""
    x, L = systems.config1()
    x = systems.jitter(x, 0.1, 3)
    args = ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 1,
            "CAL", "NAME", "QG", "STEINH", "Q", 6, "nobody", "cutoff_r", 3.9, "cutoff_Natoms", 18,
            "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "QL", "STEINH", "L", 6, "nobody", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "SYMBOL", "v1", "QG.AVE", "SYMBOL", "v2", "QL.MEAN_SOLID",
            "CV_dim", 2, "DIM", 1, 0, 1, 100, "v1", "DIM", 2, 0, 1, 100, "v2", "WT", 1]
    m = mtd.Metad(args, precision="fp64", groups={"all": 1, "nobody": 2})
    m.set_box([0, 0, 0], L)
    mask = np.ones(x.shape[0], dtype=np.int32)
    for step in range(3):
        f = np.zeros_like(x)
        m.post_force(step, np.ascontiguousarray(x), f, mask=mask)
        assert np.array_equal(m.cv, [0.0, 0.0])
        assert np.isfinite(m.compute_scalar())
        assert not np.any(f)
    m.close()


def test_zero_atoms():
    m = mtd.Metad(H.fix_args_local(), precision="mixed")
    m.set_box([0, 0, 0], [40.0, 40.0, 40.0])
    x = np.zeros((0, 3))
    f = np.zeros((0, 3))
    for step in range(2):
        m.post_force(step, x, f)
    assert np.array_equal(m.cv, [0.0, 0.0])
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_three_dimensional_grid(precision):
    """CV_dim 3 on a dense grid: WT deposits every other step, Catmull-Rom V
    and its three partial derivatives, force chain through three CVs."""
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.05, 21), L))
    args = ["GAUSSIAN", 0.05, 0.01, 9.0, "PACE", 2, "TEMP", 300.0,
            "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", 3.9,
            "CAL", "NAME", "Q4", "STEINH", "L", 4, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "CAL", "NAME", "Q6", "STEINH", "L", 6, "all", "cutoff_r", 3.9, "SW_FUNC_r", "ST",
            "CAL", "NAME", "QG", "STEINH", "Q", 6, "all", "cutoff_r", 3.9, "cutoff_Natoms", 18,
            "SYMBOL", "v1", "Q4.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID", "SYMBOL", "v3", "QG.AVE",
            "CV_dim", 3, "DIM", 1, 0, 1, 40, "v1", "DIM", 2, 0, 1, 40, "v2", "DIM", 3, 0, 1, 40, "v3", "WT", 1]
    steps = [0, 1, 2, 3]
    m, out = H.run_gpu(args, x, L, [(s, x) for s in steps], precision=precision)
    sw = O.make_sw("STEP", r0=3.9)
    o4 = O.steinh_l(4, x, L, 3.9, sw, 1e-6, None, "MEAN_SOLID")
    o6 = O.steinh_l(6, x, L, 3.9, sw, 1e-6, None, "MEAN_SOLID")
    oq = O.steinh_q(6, x, L, 3.9, 18)
    s = [o4["cv"], o6["cv"], oq["cv"]]
    g = O.Grid([[0, 1], [0, 1], [0, 1]], [40, 40, 40], 0.05, 0.01, 9.0, 300.0, 8.617343e-5, True)
    tcv, tf = TOL[precision]
    for i, step in enumerate(steps):
        if step % 2 == 0:
            g.add_hill(s)
        V, dV = g.value(s)
        cv, bias, f, _ = out[i]
        assert H.rel(cv, s) < tcv
        assert H.rel(bias, V) < tcv * 10
        fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"] + dV[2] * oq["grad"])
        assert H.rel(f, fo) < tf
    m.close()


def test_non_finite_position_fails_the_step_cleanly():
    """A NaN coordinate is flagged while binning (the atom lands in a valid
    cell and matches no neighbour test): the step deposits nothing, applies
    no bias force and reports MTD_ERR_NAN; the next good step runs normally."""
    x, L = systems.fcc(5, 5.26), np.array([5 * 5.26] * 3)
    x = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.1, 3), L))
    m = mtd.Metad(H.fix_args_local(pace=1), precision="mixed")
    m.set_box([0, 0, 0], L)
    f0 = np.full_like(x, 0.5)
    f = f0.copy()
    m.post_force(0, x, f)
    g0 = m.grid(200 * 200)
    xb = x.copy()
    xb[3, 1] = np.nan
    f = f0.copy()
    with pytest.raises(mtd.MetadError, match="non-finite"):
        m.post_force(1, xb, f)
    assert np.array_equal(f, f0)
    assert np.array_equal(m.grid(200 * 200), g0)
    f = f0.copy()
    m.post_force(2, x, f)
    assert np.all(np.isfinite(f)) and not np.array_equal(m.grid(200 * 200), g0)
    m.close()
