"""GPU parity for the structure-factor CVs, the bias grid over many steps,
HILLS output / restart, groups, virial and reproducibility."""
import os

import numpy as np
import pytest

import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu


def _fcc_jit(nc=6, seed=4, sigma=0.15):
    x, L = systems.fcc(nc, 5.26), np.array([nc * 5.26] * 3)
    return systems.jitter(x, sigma, seed), L


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["AVE", "COUNT"])
def test_debye_structure_factor(precision, mode):
    x, L = _fcc_jit(nc=7)
    sym = "SF.%s" % mode
    lo, hi, sig = (0.0, 2.0, 0.01) if mode == "AVE" else (0.0, 2000.0, 20.0)
    args = ["GAUSSIAN", sig, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "SF", "STRU_FACTOR", "all", "cutoff_r", 6.0, "q_factor", 2.8,
            "SW_func", "FERMI", "r_0", 1.0, "alpha", 5.0,
            "SYMBOL", "v1", sym, "CV_dim", 1, "DIM", 1, lo, hi, 400, "v1", "WT", 0]
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    sw = O.make_sw("FERMI", r0=1.0, alpha=5.0)
    o = O.debye(x, L, 6.0, 2.8, mode=mode, sw=sw)
    g = O.Grid([[lo, hi]], [400], sig, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([o["cv"]])
    V, dV = g.value([o["cv"]])
    cv, bias, f, _ = out[0]
    tcv, tf = (1e-9, 1e-8) if precision == "fp64" else (2e-5, 2e-3)
    assert H.rel(cv[0], o["cv"]) < tcv
    assert H.rel(f, -dV[0] * o["grad"]) < tf
    assert H.rel(m.extract("SF.stru_f", x.shape[0]), o["S"]) < tcv * 10


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_chemical_structure_factor(precision):
    """STRU_FACTOR Chemical: three atom types, Gaussian type weights around
    type 2 with a Chem_map override for type 3; CV, forces and S_i against
    the oracle.  Without types the step is refused."""
    import mtd

    x, L = _fcc_jit(nc=7)
    types = (np.arange(x.shape[0]) * 7 % 3) + 1
    args = ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "SF", "STRU_FACTOR", "all", "cutoff_r", 6.0, "q_factor", 2.8,
            "Chemical", "Chem_ctarget", 2, "Chem_sigma", 0.8, "Chem_map", "(3,0.4)",
            "SYMBOL", "v1", "SF.AVE", "CV_dim", 1, "DIM", 1, 0.0, 2.0, 400, "v1", "WT", 0]
    m = mtd.Metad(args, precision=precision)
    m.set_box([0, 0, 0], L)
    assert m.needs_types
    with pytest.raises(mtd.MetadError, match="mtd_set_types"):
        m.post_force(0, x, np.zeros_like(x))
    m.set_types(types)
    f = np.zeros_like(x)
    m.post_force(0, x, f)
    w = O.chem_type_weights(types, 2.0, 0.8, {3: 0.4})
    o = O.debye(x, L, 6.0, 2.8, weights=w)
    g = O.Grid([[0.0, 2.0]], [400], 0.01, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([o["cv"]])
    V, dV = g.value([o["cv"]])
    tcv, tf = (1e-9, 1e-8) if precision == "fp64" else (2e-5, 2e-3)
    assert H.rel(m.cv[0], o["cv"]) < tcv
    assert H.rel(f, -dV[0] * o["grad"]) < tf
    assert H.rel(m.extract("SF.stru_f", x.shape[0]), o["S"]) < tcv * 10
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("mode", ["AVE", "COUNT"])
def test_weight_chem(precision, mode):
    """WEIGHT_CHEM (type-weighted tapered pair count) against the oracle,
    with the per-atom chem_pair_r export."""
    import mtd

    x, L = _fcc_jit(nc=7)
    types = (np.arange(x.shape[0]) * 5 % 2) + 1
    sym = "CP.%s" % mode
    lo, hi, sig = (0.0, 40.0, 0.2) if mode == "AVE" else (0.0, 1000.0, 10.0)
    args = ["GAUSSIAN", sig, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "CP", "WEIGHT_CHEM", "all", "cutoff_r", 4.5, "Chem_map", "(1,0.1)", "(2", "3.0)",
            "SW_func", "FERMI", "r_0", 30.0, "alpha", 0.1,
            "SYMBOL", "v1", sym, "CV_dim", 1, "DIM", 1, lo, hi, 400, "v1", "WT", 0]
    m = mtd.Metad(args, precision=precision)
    m.set_box([0, 0, 0], L)
    m.set_types(types)
    f = np.zeros_like(x)
    m.post_force(0, x, f)
    w = O.chem_type_weights(types, cmap={1: 0.1, 2: 3.0})
    o = O.debye(x, L, 4.5, 0.0, mode=mode, sw=O.make_sw("FERMI", r0=30.0, alpha=0.1), weights=w)
    g = O.Grid([[lo, hi]], [400], sig, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([o["cv"]])
    V, dV = g.value([o["cv"]])
    tcv, tf = (1e-9, 1e-8) if precision == "fp64" else (2e-5, 2e-3)
    assert H.rel(m.cv[0], o["cv"]) < tcv
    assert H.rel(f, -dV[0] * o["grad"]) < tf
    assert H.rel(m.extract("CP.chem_pair_r", x.shape[0]), o["S"]) < tcv * 10
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_kvector_structure_factor(precision):
    x, L = _fcc_jit(nc=8, sigma=0.2)
    kvec = systems.kvectors(24, systems.KMAG_111, 99)
    args = ["GAUSSIAN", 0.5, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "SK", "STRU_FACTOR_K", "all", "nk", 24, "kmag", systems.KMAG_111, "seed", 99,
            "SYMBOL", "v1", "SK.AVE", "CV_dim", 1, "DIM", 1, 0.0, 100.0, 500, "v1", "WT", 0]
    m, out = H.run_gpu(args, x, L, [(0, x)], precision=precision)
    o = O.sk(x, kvec)
    g = O.Grid([[0.0, 100.0]], [500], 0.5, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([o["cv"]])
    V, dV = g.value([o["cv"]])
    cv, bias, f, _ = out[0]
    tcv, tf = (1e-9, 1e-8) if precision == "fp64" else (1e-5, 1e-4)
    assert H.rel(cv[0], o["cv"]) < tcv
    assert H.rel(f, -dV[0] * o["grad"]) < tf


def test_kvector_structure_factor_full_size():
    """1,048,576 atoms, 96 k-vectors on the first FCC Bragg shell: mixed mode
    against the FP64 oracle (S 1e-5, forces 1e-4 of the largest component)."""
    x, L = systems.config3()
    kvec = systems.kvectors(96, systems.KMAG_111, 3)
    args = ["GAUSSIAN", 0.05, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "SK", "STRU_FACTOR_K", "all", "nk", 96, "kmag", systems.KMAG_111, "seed", 3,
            "SYMBOL", "v1", "SK.AVE", "CV_dim", 1, "DIM", 1, 0.0, 10.0, 2000, "v1", "WT", 0]
    m, out = H.run_gpu(args, x, L, [(0, x)], precision="mixed")
    o = O.sk(x, kvec)
    g = O.Grid([[0.0, 10.0]], [2000], 0.05, 0.005, 10.0, 300.0, 8.617343e-5, False)
    g.add_hill([o["cv"]])
    V, dV = g.value([o["cv"]])
    cv, bias, f, _ = out[0]
    assert H.rel(cv[0], o["cv"]) < 1e-5
    assert H.rel(bias, V) < 1e-5
    assert H.rel(f, -dV[0] * o["grad"]) < 1e-4


def test_grid_many_steps_matches_oracle():
    """C1 protocol on 30 steps: jittered FCC re-drawn every step, PACE 10, WT 1;
    the whole 1000-bin grid is compared after the run."""
    x0, L = systems.config1()
    args = H.fix_args_q(wt=1, pace=10)
    m = mtd.Metad(args, precision="fp64")
    m.set_box([0, 0, 0], L)
    g = O.Grid([[0.0, 1.0]], [1000], 0.01, 0.005, 10.0, 300.0, 8.617343e-5, True)
    for step in range(0, 31):
        x = systems.jitter(x0, 0.15, 17, step)
        f = np.zeros_like(x)
        m.post_force(step, x, f)
        o = O.steinh_q(6, x, L, 3.9, 18)
        if step % 10 == 0:
            g.add_hill([o["cv"]])
        V, dV = g.value([o["cv"]])
        assert abs(m.cv[0] - o["cv"]) < 1e-12
        assert abs(m.compute_scalar() - V) < 1e-12 + 1e-10 * abs(V)
        assert H.rel(f, -dV[0] * o["grad"]) < 1e-9
    grid = m.grid(1000)
    assert np.max(np.abs(grid - g.grid)) < 1e-12


def test_hills_file_and_restart(tmp_path):
    x0, L = systems.config1()
    hills = str(tmp_path / "HILLS")
    args = H.fix_args_q(wt=1, pace=5)
    m = mtd.Metad(args, precision="fp64", hills_path=hills)
    m.set_box([0, 0, 0], L)
    for step in range(0, 21):
        x = systems.jitter(x0, 0.15, 3, step)
        m.post_force(step, x, np.zeros_like(x))
    grid1 = m.grid(1000)
    m.close()
    lines = open(hills).read().splitlines()
    assert lines[0] == "# step cv_values height sigma"
    rows = [ln.split() for ln in lines[1:]]
    assert [int(r[0]) for r in rows] == [0, 5, 10, 15, 20]
    assert all(len(r) == 4 for r in rows)
    # restart: METAD_RESTART 1 replays the file into an identical grid and appends
    m2 = mtd.Metad(args + ["METAD_RESTART", 1], precision="fp64", hills_path=hills)
    m2.set_box([0, 0, 0], L)
    m2.init()
    grid2 = m2.grid(1000)
    assert np.max(np.abs(grid2 - grid1)) < 1e-12
    x = systems.jitter(x0, 0.15, 3, 25)
    m2.post_force(25, x, np.zeros_like(x))
    m2.close()
    lines2 = open(hills).read().splitlines()
    assert len(lines2) == len(lines) + 1 and lines2[-1].startswith("25 ")


@pytest.mark.parametrize("bad", ["10 0.25 0.005\n", "10 0.25 abc 0.01\n", "ten 0.25 0.005 0.01\n"])
def test_corrupt_hills_line_is_an_error(tmp_path, bad):
    """A truncated or non-numeric HILLS row stops the restart with
    MTD_ERR_IO and the offending line, before any step (comment and blank
    lines are skipped)."""
    hills = tmp_path / "HILLS"
    hills.write_text("# step cv_values height sigma\n\n0 0.20 0.005 0.01\n" + bad)
    m = mtd.Metad(H.fix_args_q(wt=1, pace=5) + ["METAD_RESTART", 1], precision="fp64", hills_path=str(hills))
    m.set_box([0, 0, 0], [20.0, 20.0, 20.0])
    with pytest.raises(mtd.MetadError, match="malformed HILLS line"):
        m.init()
    m.close()


def test_empty_hills_file_restarts_fresh_with_a_header(tmp_path):
    """METAD_RESTART 1 with an existing but empty HILLS file: nothing to
    replay, the file is rewritten with its header (not appended to without
    one), and the first deposit lands below the header."""
    x0, L = systems.config1()
    hills = tmp_path / "HILLS"
    hills.write_text("")
    m = mtd.Metad(H.fix_args_q(wt=1, pace=5) + ["METAD_RESTART", 1], precision="fp64", hills_path=str(hills))
    m.set_box([0, 0, 0], L)
    m.init()
    assert np.all(m.grid(1000) == 0.0)
    x = systems.jitter(x0, 0.15, 3, 0)
    m.post_force(0, x, np.zeros_like(x))
    m.close()
    lines = hills.read_text().splitlines()
    assert lines[0] == "# step cv_values height sigma" and len(lines) == 2 and lines[1].startswith("0 ")


def test_reference_hills_fixture_replays():
    """The reference's own 1D HILLS (test/test_cvset/HILLS: 238 hills, h 0.005,
    sigma 0.01), committed under tests/golden, replays like the oracle's sum."""
    path = os.path.join(os.path.dirname(__file__), "golden", "HILLS_1d_reference_fixture")
    if not os.path.exists(path):
        pytest.skip("fixture not generated")
    rows = np.array([[float(t) for t in ln.split()] for ln in open(path) if ln.strip() and ln[0] != "#"])
    args = H.fix_args_q(nbins=1000)
    m = mtd.Metad(args, precision="fp64")
    m.set_box([0, 0, 0], [52.6] * 3)
    m.init()
    m.hills_replay(path)
    g = O.Grid([[0.0, 1.0]], [1000], 0.01, 0.005, 10.0, 300.0, 8.617343e-5, False)
    for r in rows:
        g.deposit([r[1]], r[2], sigma=r[3])
    assert np.max(np.abs(m.grid(1000) - g.grid)) < 1e-13


def test_group_mask_and_virial():
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = systems.jitter(x, 0.05, 9)
    n = x.shape[0]
    mask = np.where(np.arange(n) % 3 == 0, 1, 1 | 2).astype(np.int32)   # "all" = 1, "sub" = 2
    args = H.fix_args_local()
    for l in (4, 6):
        i = args.index("Q%d" % l, args.index("CAL"))
        args[i + 4] = "sub"
    groups = {"all": 1, "sub": 2}
    m, out = H.run_gpu(args, x, L, [(0, x)], precision="fp64", groups=groups, mask=mask, virial=True)
    ing = ((mask & 2) != 0).astype(np.int32)
    o4 = H.oracle_local(x, L, 4, ingroup=ing)
    o6 = H.oracle_local(x, L, 6, ingroup=ing)
    g = O.Grid([[0, 1], [0, 1]], [200, 200], 0.01, 0.005, 9.0, 300.0, 8.617343e-5, True)
    s = [o4["cv"], o6["cv"]]
    g.add_hill(s)
    V, dV = g.value(s)
    fo = -(dV[0] * o4["grad"] + dV[1] * o6["grad"])
    cv, bias, f, vir = out[0]
    assert H.rel(cv, s) < 1e-9
    assert H.rel(f, fo) < 1e-8
    vo = np.array([np.sum(fo[:, 0] * x[:, 0]), np.sum(fo[:, 1] * x[:, 1]), np.sum(fo[:, 2] * x[:, 2]),
                   np.sum(fo[:, 0] * x[:, 1]), np.sum(fo[:, 0] * x[:, 2]), np.sum(fo[:, 1] * x[:, 2])])
    assert H.rel(vir, vo) < 1e-8


def test_out_of_range_cv_is_safe():
    """A CV far outside the DIM range deposits nothing and yields finite forces."""
    x, L = _fcc_jit(nc=5)
    args = H.fix_args_q(lo=5.0, hi=6.0, nbins=100)
    m, out = H.run_gpu(args, x, L, [(0, x), (10, x)], precision="fp64")
    assert np.all(m.grid(100) == 0.0)
    for cv, bias, f, _ in out:
        assert np.all(np.isfinite(f)) and bias == 0.0


def test_reproducible_bitwise_and_translation_invariant():
    """Two contexts give bitwise-identical results; forces sum to ~0 (the CVs are
    translation invariant) on the full 256k-atom slab system."""
    x, L = systems.config2()
    x = systems.wrap(systems.jitter(x, 0.05, 1), L)
    args = H.fix_args_local()
    res = []
    for _ in range(2):
        m, out = H.run_gpu(args, x, L, [(0, x), (10, x)], precision="mixed")
        res.append(out)
        assert m.max_neighbors("Q4") <= 18
        m.close()
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a[0], b[0]) and a[1] == b[1] and np.array_equal(a[2], b[2])
    f = res[0][1][2]
    assert np.abs(f.sum(axis=0)).max() < 1e-4 * np.abs(f).max() * np.sqrt(x.shape[0])
