"""Domain decomposition through the C ABI on one GPU: two ranks emulated as
two contexts driven by two host threads (each with its own stream; they meet
only on the host, in the allreduce callback), against one context holding the
whole periodic system.  Forces are compared after the ghost rows have been
added to their owners; CVs, bias and the grid must agree with the single
domain, and bit for bit between the ranks."""
import threading

import numpy as np
import pytest

import domain
import helpers as H
import mtd
import oracle as O
import systems

pytestmark = pytest.mark.gpu


def _fcc(nc=7, seed=4, sigma=0.15):
    x, L = systems.fcc(nc, 5.26), np.array([nc * 5.26] * 3)
    return systems.wrap(systems.jitter(x, sigma, seed), L), L


def _args_q():
    return ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 1, "TEMP", 300.0,
            "CAL", "NAME", "SWC", "SW_FUNC", "FERMI", "r_0", 0.45, "alpha", 20.0,
            "CAL", "NAME", "Q6", "STEINH", "Q", 6, "all", "cutoff_r", 4.5, "cutoff_Natoms", 12,
            "SYMBOL", "v1", "Q6.AVE", "SYMBOL", "v2", "Q6.SW_FUNC.SWC", "CV_dim", 2,
            "DIM", 1, 0.0, 1.0, 200, "v1", "DIM", 2, 0.0, 2000.0, 200, "v2", "WT", 1]


def _args_sf():
    return ["GAUSSIAN", 20.0, 0.005, 10.0, "PACE", 1,
            "CAL", "NAME", "SF", "STRU_FACTOR", "all", "cutoff_r", 6.0, "q_factor", 2.8, "Chemical",
            "Chem_ctarget", 2.0, "Chem_sigma", 0.8, "Chem_map", "(3,0.4)",
            "SW_func", "FERMI", "r_0", 1.0, "alpha", 5.0,
            "SYMBOL", "v1", "SF.COUNT", "CV_dim", 1, "DIM", 1, 0.0, 2000.0, 400, "v1", "WT", 0]


def _args_sk(nk=24):
    return ["GAUSSIAN", 0.01, 0.005, 10.0, "PACE", 1,
            "CAL", "NAME", "SK", "STRU_FACTOR_K", "all", "nk", nk, "kmag", systems.KMAG_111, "seed", 3,
            "SYMBOL", "v1", "SK.AVE", "CV_dim", 1, "DIM", 1, 0.0, 2.0, 400, "v1", "WT", 0]


CASES = {
    "steinh_l_step": lambda: H.fix_args_local(pace=1),
    "steinh_l_fermi": lambda: H.fix_args_local(pace=1, sw="FERMI"),
    "steinh_q": _args_q,
    "stru_factor_chem": _args_sf,
    "sk": _args_sk,
}


def _run_single(args, x, L, steps, precision, types, tmp):
    m = mtd.Metad(args, precision=precision, hills_path="HILLS", work_dir=str(tmp))
    m.set_box([0, 0, 0], L)
    if m.needs_types:
        m.set_types(types)
    out = []
    for step, xs in steps:
        f = np.zeros_like(xs)
        m.post_force(step, xs, f)
        out.append((m.cv, m.compute_scalar(), f))
    grid = m.grid(_grid_size(args))
    m.close()
    return out, grid


def _grid_size(args):
    a = [str(t) for t in args]
    size, i = 1, 0
    while i < len(a):
        if a[i] == "DIM":
            size *= int(a[i + 4])
            i += 5
        else:
            i += 1
    return size


def _run_ranks(args, x, L, steps, precision, types, tmp, grid=(2, 1, 1)):
    probe = mtd.Metad(args, precision=precision)
    cut = probe.ghost_cutoff
    probe.close()
    nr = int(np.prod(grid))
    red = domain.LocalAllreduce(nr, timeout=120)
    ctx = []
    for r in range(nr):
        m = mtd.Metad(args, precision=precision, hills_path="HILLS", work_dir=str(tmp))
        m.set_domain(0, r, red.for_rank(r))
        ctx.append(m)
    res = [[None] * len(steps) for _ in range(nr)]
    errs = []

    def run(r):
        try:
            m = ctx[r]
            for s, (step, xs) in enumerate(steps):
                rk = domain.decompose(xs, [0, 0, 0], L, grid, max(cut, 1e-9))[r]
                m.set_box(rk["lo"], rk["hi"], (0, 0, 0))
                m.set_nlocal(rk["owned"].size)
                if m.needs_types:
                    m.set_types(types[rk["ids"]])
                f = np.zeros_like(rk["x"])
                m.post_force(step, rk["x"], f)
                res[r][s] = (m.cv, m.compute_scalar(), f, rk)
        except BaseException as e:   # the other rank's barrier gives up instead of waiting
            errs.append(e)
            red.abort()

    ts = [threading.Thread(target=run, args=(r,)) for r in range(nr)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    if errs:
        raise errs[0]
    grids = [m.grid(_grid_size(args)) for m in ctx]
    for m in ctx:
        m.close()
    return res, grids, cut


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("case", list(CASES))
def test_two_ranks_equal_one_domain(case, precision, tmp_path):
    args = CASES[case]()
    x, L = _fcc()
    n = x.shape[0]
    types = (np.arange(n) * 7 % 4).astype(np.int32)
    steps = [(s, np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.03, 90, s), L))) for s in range(3)]
    (tmp_path / "one").mkdir()
    (tmp_path / "two").mkdir()
    single, grid1 = _run_single(args, x, L, steps, precision, types, tmp_path / "one")
    ranks, grids, cut = _run_ranks(args, x, L, steps, precision, types, tmp_path / "two")
    # 2 x the STEINH L list radius: r_0 for STEP, sigma(r) = cutoff_eps for FERMI
    rl = O.sw_invert_for_eps(O.make_sw("FERMI", r0=3.9, alpha=-8.0), 1e-6)
    assert cut == pytest.approx({"steinh_l_step": 7.8, "steinh_l_fermi": 2 * rl, "steinh_q": 4.5,
                                 "stru_factor_chem": 6.0, "sk": 0.0}[case])
    tcv, tf = (1e-10, 1e-8) if precision == "fp64" else (2e-5, 3e-3)
    for s in range(len(steps)):
        cv1, b1, f1 = single[s]
        for r in range(2):
            cv, b, _, _ = ranks[r][s]
            assert np.array_equal(cv, ranks[0][s][0]) and b == ranks[0][s][1]
            assert H.rel(cv, cv1) < tcv
            assert H.rel(b, b1) < max(tcv, 1e-9)
        f = domain.reverse_sum(n, [ranks[r][s][3] for r in range(2)], [ranks[r][s][2] for r in range(2)])
        assert H.rel(f, f1) < tf
    assert np.array_equal(grids[0], grids[1])
    assert H.rel(grids[0], grid1) < max(tcv, 1e-9)
    rows = [l for l in (tmp_path / "two" / "HILLS").read_text().splitlines() if not l.startswith("#")]
    assert len(rows) == len(steps)   # rank 0 alone writes HILLS


@pytest.mark.parametrize("case", ["steinh_l_step", "stru_factor_chem"])
def test_four_ranks_in_a_2x2_grid(case, tmp_path):
    """Four thread ranks over a 2 x 2 x 1 brick grid (ghosts from two
    neighbouring bricks and their corner), FP64, against one domain."""
    args = CASES[case]()
    x, L = _fcc(nc=8)
    n = x.shape[0]
    types = (np.arange(n) * 7 % 4).astype(np.int32)
    steps = [(s, np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.03, 91, s), L))) for s in range(2)]
    (tmp_path / "one").mkdir()
    (tmp_path / "four").mkdir()
    single, grid1 = _run_single(args, x, L, steps, "fp64", types, tmp_path / "one")
    ranks, grids, _ = _run_ranks(args, x, L, steps, "fp64", types, tmp_path / "four", grid=(2, 2, 1))
    for s in range(len(steps)):
        cv1, b1, f1 = single[s]
        for r in range(4):
            assert np.array_equal(ranks[r][s][0], ranks[0][s][0]) and ranks[r][s][1] == ranks[0][s][1]
        assert H.rel(ranks[0][s][0], cv1) < 1e-10 and H.rel(ranks[0][s][1], b1) < 1e-9
        f = domain.reverse_sum(n, [ranks[r][s][3] for r in range(4)], [ranks[r][s][2] for r in range(4)])
        assert H.rel(f, f1) < 1e-8
    for g in grids[1:]:
        assert np.array_equal(g, grids[0])
    assert H.rel(grids[0], grid1) < 1e-9


def test_overflow_on_one_rank_retries_on_every_rank(tmp_path):
    """A dense cluster inside rank 0's brick overflows its neighbour lists on
    the first step while rank 1's do not: the overflow flag travels with the
    totals, both ranks skip the deposit and retry together, and the result
    equals the single domain (which overflows and retries too)."""
    x, L = _fcc(nc=7)
    rng = np.random.default_rng(5)
    c = np.array([0.25, 0.5, 0.5]) * L
    blob = c + rng.uniform(-1.2, 1.2, size=(40, 3))
    x = np.ascontiguousarray(np.concatenate([x, blob]))
    n = x.shape[0]
    types = np.ones(n, dtype=np.int32)
    args = CASES["steinh_l_step"]()
    steps = [(s, x) for s in range(2)]
    (tmp_path / "one").mkdir()
    (tmp_path / "two").mkdir()
    single, grid1 = _run_single(args, x, L, steps, "fp64", types, tmp_path / "one")
    ranks, grids, _ = _run_ranks(args, x, L, steps, "fp64", types, tmp_path / "two")
    for s in range(len(steps)):
        cv1, b1, f1 = single[s]
        assert np.array_equal(ranks[0][s][0], ranks[1][s][0])
        assert H.rel(ranks[0][s][0], cv1) < 1e-10 and H.rel(ranks[0][s][1], b1) < 1e-9
        f = domain.reverse_sum(n, [ranks[r][s][3] for r in range(2)], [ranks[r][s][2] for r in range(2)])
        assert H.rel(f, f1) < 1e-8
    assert np.array_equal(grids[0], grids[1]) and H.rel(grids[0], grid1) < 1e-9


def _one_rank_vs_plain(setup, precision="mixed"):
    """A single rank owning every atom of the periodic box, exchange through
    `setup(m)`, against the plain context: the same bits (the one-rank sum
    is the rank's own totals, reduced in the bias kernel's order)."""
    x, L = _fcc(nc=6)
    args = H.fix_args_local(pace=1)
    a = mtd.Metad(args, precision=precision)
    b = mtd.Metad(args, precision=precision)
    setup(b, x.shape[0])
    for m in (a, b):
        m.set_box([0, 0, 0], L)
    for s in range(3):
        xs = np.ascontiguousarray(systems.wrap(systems.jitter(x, 0.03, 95, s), L))
        fa, fb = np.zeros_like(xs), np.zeros_like(xs)
        a.post_force(s, xs, fa)
        b.post_force(s, xs, fb)
        assert np.array_equal(fa, fb) and np.array_equal(a.cv, b.cv) and a.compute_scalar() == b.compute_scalar()
    a.close()
    b.close()


def test_device_exchange_one_rank_identity():
    """Device-side exchange with a callback that enqueues nothing (the sum
    over one rank): no host round trip, same bits as the plain step."""
    calls = []
    _one_rank_vs_plain(lambda m, n: m.set_domain_device(n, 0, lambda p, c, s: calls.append((c, s))))
    assert len(calls) == 3 and all(c == calls[0][0] for c, _ in calls)


def test_device_exchange_one_rank_nccl():
    """Device-side exchange through torch.distributed NCCL (world size 1),
    enqueued on the library's stream."""
    import socket

    import torch.distributed as dist
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        _one_rank_vs_plain(lambda m, n: m.set_domain_device(n, 0, domain.TorchDeviceAllreduce()))
    finally:
        dist.destroy_process_group()


def test_domain_api_errors():
    m = mtd.Metad(H.fix_args_local())
    with pytest.raises(mtd.MetadError, match="domain decomposition is not enabled"):
        m.set_nlocal(10)
    red = domain.LocalAllreduce(1)
    m.set_domain(5, 0, red.for_rank(0))
    x, L = _fcc(nc=3)
    m.set_box([0, 0, 0], L, (0, 0, 0))
    m.set_nlocal(x.shape[0] + 1)
    with pytest.raises(mtd.MetadError, match="exceeds"):
        m.post_force(0, x, np.zeros_like(x))
    m.close()
    m = mtd.Metad(H.fix_args_local())
    m.set_box([0, 0, 0], L)
    m.post_force(0, x, np.zeros_like(x))
    with pytest.raises(mtd.MetadError, match="before the first step"):
        m.set_domain(5, 0, red.for_rank(0))
    m.close()


def test_non_finite_position_on_one_rank_stops_every_rank(tmp_path):
    """A NaN coordinate among rank 0's owned atoms: the non-finite flag travels
    with the totals, so neither rank deposits or applies a bias force, both
    report MTD_ERR_NAN for that step (a LAMMPS error->all() is then reached by
    every rank), the replicated grids stay equal, and the next good step runs
    on both ranks."""
    args = CASES["steinh_l_step"]()
    x, L = _fcc(nc=7)
    probe = mtd.Metad(args, precision="mixed")
    cut = probe.ghost_cutoff
    probe.close()
    red = domain.LocalAllreduce(2, timeout=120)
    ctx = []
    for r in range(2):
        m = mtd.Metad(args, precision="mixed", hills_path="HILLS", work_dir=str(tmp_path))
        m.set_domain(0, r, red.for_rank(r))
        ctx.append(m)
    status = [[None] * 3 for _ in range(2)]
    forces = [[None] * 3 for _ in range(2)]
    grids = [[None] * 3 for _ in range(2)]
    errs = []

    def run(r):
        try:
            m = ctx[r]
            for step in range(3):
                rk = domain.decompose(x, [0, 0, 0], L, (2, 1, 1), cut)[r]
                xr = rk["x"].copy()
                if step == 1 and r == 0:
                    xr[0, 1] = np.nan
                m.set_box(rk["lo"], rk["hi"], (0, 0, 0))
                m.set_nlocal(rk["owned"].size)
                f0 = np.full_like(xr, 0.25)
                f = f0.copy()
                try:
                    m.post_force(step, xr, f)
                    status[r][step] = "ok"
                except mtd.MetadError as e:
                    status[r][step] = "nan" if "non-finite" in str(e) else str(e)
                forces[r][step] = np.array_equal(f, f0)
                grids[r][step] = m.grid(200 * 200)
        except BaseException as e:
            errs.append(e)
            red.abort()

    ts = [threading.Thread(target=run, args=(r,)) for r in range(2)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    for m in ctx:
        m.close()
    if errs:
        raise errs[0]
    assert status[0] == ["ok", "nan", "ok"] and status[1] == ["ok", "nan", "ok"]
    assert forces[0][1] and forces[1][1]              # no bias force on either rank at the bad step
    assert not forces[0][2] and not forces[1][2]      # the next step applies it again
    for s in range(3):
        assert np.array_equal(grids[0][s], grids[1][s])
    assert np.array_equal(grids[0][1], grids[0][0])   # nothing deposited at the bad step
    assert not np.array_equal(grids[0][2], grids[0][1])
