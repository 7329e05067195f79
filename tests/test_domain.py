"""Domain decomposition on CPU: the host-side split into owned atoms and ghost
images (metad-toy_b200/domain.py), the allreduce helpers, and -- with two
gloo ranks -- the decomposed CVs and gradients of the oracle against the
undecomposed ones.  Each rank evaluates its owned atoms as centres (group 1)
and its ghosts as neighbours only (group 0), sums its totals with the other
rank through the same allreduce callback the library calls, and adds its
ghost gradient rows to their owners; the result must equal the single-domain
oracle.  The ghost shell is cutoff_r for STEINH Q and STRU_FACTOR and 2 x
cutoff for STEINH L, the rule of mtd_ghost_cutoff."""
import datetime
import os
import socket
import sys
import threading

import numpy as np
import pytest
import torch.multiprocessing as mp

import domain
import oracle as O
import systems

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _system(nc=5, seed=11):
    x, L = systems.fcc(nc, 5.26), np.array([nc * 5.26] * 3)
    return systems.wrap(systems.jitter(x, 0.15, seed), L), L


def _minimg_pairs(x, L, rc):
    d = x[None, :, :] - x[:, None, :]
    d -= L * np.rint(d / L)
    r2 = np.einsum("ijk,ijk->ij", d, d)
    np.fill_diagonal(r2, np.inf)
    return r2 <= rc * rc, d


@pytest.mark.parametrize("grid", [(2, 1, 1), (2, 2, 1), (1, 1, 3)])
def test_decompose_reproduces_every_neighbourhood(grid):
    """Every owned atom sees, among its rank's owned + ghost rows, exactly its
    periodic neighbours within the ghost cutoff, at the same displacements."""
    x, L = _system(nc=4)
    cut = 4.0
    ranks = domain.decompose(x, [0, 0, 0], L, grid, cut)
    owned_all = np.sort(np.concatenate([r["owned"] for r in ranks]))
    assert np.array_equal(owned_all, np.arange(x.shape[0]))
    near, disp = _minimg_pairs(x, L, cut)
    for r in ranks:
        xl, ids = r["x"], r["ids"]
        assert np.all(xl >= r["lo"]) and np.all(xl < r["hi"])
        for a, i in enumerate(r["owned"]):
            dl = xl - xl[a]
            sel = np.nonzero(np.einsum("ij,ij->i", dl, dl) <= cut * cut)[0]
            sel = sel[sel != a]
            got = sorted((int(ids[b]), *np.round(dl[b], 9)) for b in sel)
            want = sorted((int(j), *np.round(disp[i, j], 9)) for j in np.nonzero(near[i])[0])
            assert got == want


def test_reverse_sum_adds_ghost_rows_to_owners():
    x, L = _system(nc=3)
    ranks = domain.decompose(x, [0, 0, 0], L, (2, 1, 1), 3.0)
    rows = [np.ones((r["ids"].size, 3)) for r in ranks]
    tot = domain.reverse_sum(x.shape[0], ranks, rows)
    copies = np.zeros(x.shape[0])
    for r in ranks:
        np.add.at(copies, r["ids"], 1.0)
    assert np.array_equal(tot[:, 0], copies)


def test_local_allreduce_gives_every_rank_the_same_sum():
    n = 3
    red = domain.LocalAllreduce(n, timeout=30)
    bufs = [np.arange(5, dtype=np.float64) * (r + 1) + 0.1 * r for r in range(n)]
    ts = [threading.Thread(target=red.for_rank(r), args=(bufs[r],)) for r in range(n)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    want = sum(np.arange(5, dtype=np.float64) * (r + 1) + 0.1 * r for r in range(n))
    for b in bufs:
        assert np.array_equal(b, bufs[0]) and np.allclose(b, want)


def _cases():
    """(name, ghost shell, oracle call on (x, L, periodic, ingroup)), the
    linear CVs (COUNT / SW sums, and AVE through its count)."""
    fermi = O.make_sw("FERMI", r0=0.45, alpha=20.0)
    swr = O.make_sw("FERMI", r0=3.9, alpha=-8.0)
    kv = systems.kvectors(8, 2 * np.pi / 3.72, 3)
    return [
        ("debye_count", 6.0, lambda x, L, p, g: O.debye(x, L, 6.0, 2.8, mode="COUNT",
                                                        sw=O.make_sw("FERMI", r0=1.0, alpha=5.0),
                                                        ingroup=g, periodic=p)),
        ("q6_ave", 4.5, lambda x, L, p, g: O.steinh_q(6, x, L, 4.5, 12, ingroup=g, periodic=p)),
        ("q6_sw", 4.5, lambda x, L, p, g: O.steinh_q(6, x, L, 4.5, 12, mode="SW_FUNC", swcv=fermi,
                                                     ingroup=g, periodic=p)),
        ("l6_nsolid", 2 * 4.6, lambda x, L, p, g: O.steinh_l(6, x, L, 4.6, swr, swcv=fermi, mode="NSOLID",
                                                             ingroup=g, periodic=p)),
        ("sk", 0.0, lambda x, L, p, g: O.sk(x, kv, ingroup=g)),
    ]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    for p in (os.path.join(ROOT, "metad-toy_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    import test_domain as T
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        red = domain.TorchAllreduce()
        x, L = T._system()
        n = x.shape[0]
        res = {}
        for name, shell, fn in T._cases():
            rk = domain.decompose(x, [0, 0, 0], L, (world, 1, 1), max(shell, 1e-9))[rank]
            nl = rk["owned"].size
            g = np.zeros(rk["ids"].size, dtype=np.int32)
            g[:nl] = 1
            o = fn(rk["x"], rk["hi"] - rk["lo"], (0, 0, 0), g)
            if name == "sk":   # S(k) is quadratic in rho(k): the ranks sum rho(k) and N (no ghosts needed)
                buf = np.concatenate([o["rho"].reshape(-1), [float(nl)]])
                red(buf)
                rho = buf[:-1].reshape(-1, 2)
                res[name] = (float(np.sum(rho * rho)) / buf[-1] / rho.shape[0], None)
                continue
            ave = name.endswith("_ave")
            buf = np.array([o["cv"] * nl if ave else o["cv"], float(nl)])
            red(buf)
            cv = buf[0] / buf[1] if ave else buf[0]
            grow = np.zeros((n, 3))
            np.add.at(grow, rk["ids"], o["grad"] * (nl / n if ave else 1.0))
            flat = grow.reshape(-1).copy()
            red(flat)
            res[name] = (cv, flat.reshape(n, 3))
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_match_the_single_domain_oracle():
    world = 2
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    x, L = _system()
    ref = {name: fn(x, L, (1, 1, 1), None) for name, _, fn in _cases()}
    for name, o in ref.items():
        for rank in range(world):
            cv, grad = res[rank][name]
            assert cv == pytest.approx(o["cv"], rel=1e-12, abs=1e-12), name
            if grad is None:
                continue
            scale = max(1e-30, np.abs(o["grad"]).max())
            assert np.abs(grad - o["grad"]).max() / scale < 1e-10, name
        assert res[0][name][0] == res[1][name][0]


def test_local_allgather_orders_by_rank():
    n = 3
    red = domain.LocalAllgather(n, timeout=30)
    sends = [np.full(4, float(r + 1)) for r in range(n)]
    recvs = [np.zeros(4 * n) for _ in range(n)]
    ts = [threading.Thread(target=red.for_rank(r), args=(sends[r], recvs[r])) for r in range(n)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    want = np.concatenate(sends)
    for rv in recvs:
        assert np.array_equal(rv, want)
