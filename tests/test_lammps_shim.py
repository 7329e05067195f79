"""The LAMMPS shim (metad-toy_b200/lammps: fix metad, compute metad/atom and
the plugin registration) against stand-in LAMMPS classes (tests/lammps_stub):
it compiles against the API it uses, and driven like LAMMPS drives a fix
(plugin load, fix and compute from deck tokens, init, post_force with the
virial flag each step) it gives exactly the library's own step: same forces
bit for bit, bias, CVs, virial and per-atom exports.  On two ranks (host
threads with their own LAMMPS instances; MPI_Allreduce and reverse
communication served across them) the fix equals the library's own
domain-decomposed step."""
import os
import struct
import subprocess
import threading

import numpy as np
import pytest

import helpers as H

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "metad-toy_b200")
SRCS = [os.path.join(ROOT, "tests", "lammps_stub", "harness.cpp")] + [
    os.path.join(PKG, "lammps", f) for f in ("fix_metad_b200.cpp", "compute_metad_atom_b200.cpp", "plugin_b200.cpp")]


def _build(tmp_path):
    exe = str(tmp_path / "harness")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I" + os.path.join(ROOT, "tests", "lammps_stub"),
           "-I" + os.path.join(ROOT, "include"), "-I" + os.path.join(PKG, "lammps")] + SRCS + [
        "-L" + PKG, "-lmetad_b200", "-Wl,-rpath," + PKG, "-lpthread", "-o", exe]
    subprocess.check_call(cmd)
    return exe


def test_shim_compiles_against_the_lammps_api(tmp_path):
    assert os.path.exists(_build(tmp_path))


@pytest.mark.gpu
def test_shim_step_equals_library_step(tmp_path):
    import mtd
    import systems

    exe = _build(tmp_path)
    x0, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x0, 0.05, 60, s), L)) for s in range(4)]
    n = x0.shape[0]
    mask = np.ones(n, dtype=np.int32)
    args = [str(a) for a in H.fix_args_local(pace=2)]
    reqs = ["Q4.stein_q", "Q6.dcvdx_x"]
    with open(tmp_path / "in.bin", "wb") as fh:
        fh.write(struct.pack("ii", n, len(xs)))
        fh.write(np.zeros(3).tobytes() + np.asarray(L, dtype=np.float64).tobytes())
        fh.write(np.array([1, 1, 1], dtype=np.int32).tobytes())
        for x in xs:
            fh.write(x.tobytes())
        fh.write(mask.tobytes())
    with open(tmp_path / "tokens.txt", "w") as fh:
        fh.write("\n".join(args + ["--"] + reqs) + "\n")
    subprocess.check_call([exe, str(tmp_path / "in.bin"), str(tmp_path / "tokens.txt"), str(tmp_path / "out.bin")],
                          cwd=str(tmp_path))
    raw = np.fromfile(tmp_path / "out.bin", dtype=np.float64)

    m = mtd.Metad(args, precision="mixed", work_dir=str(tmp_path))
    m.set_box([0, 0, 0], L)
    off, D = 0, 2
    for step, x in enumerate(xs):
        f = np.zeros_like(x)
        vir = m.post_force(step, x, f, virial=True)
        bias, cv = raw[off], raw[off + 1:off + 1 + D]
        v6 = raw[off + 1 + D:off + 7 + D]
        fs = raw[off + 7 + D:off + 7 + D + 3 * n].reshape(n, 3)
        off += 7 + D + 3 * n
        assert bias == m.compute_scalar() and np.array_equal(cv, m.cv)
        assert np.array_equal(v6, vir) and np.array_equal(fs, f)
    per = raw[off:].reshape(n, len(reqs))
    assert np.array_equal(per[:, 0], m.extract("Q4.stein_q", n))
    assert np.array_equal(per[:, 1], m.extract("Q6.dcvdx_x", n))
    m.close()


def _write_rank(path, gc, steps):
    with open(path, "wb") as fh:
        fh.write(struct.pack("i", len(steps)) + struct.pack("d", gc))
        for st in steps:
            nl, ng = st["nlocal"], st["grank"].size
            fh.write(struct.pack("ii", nl, ng))
            fh.write(np.asarray(st["sublo"], dtype=np.float64).tobytes() + np.asarray(st["subhi"], dtype=np.float64).tobytes())
            fh.write(np.ascontiguousarray(st["x"]).tobytes())
            fh.write(np.ones(nl + ng, dtype=np.int32).tobytes())
            fh.write(np.ascontiguousarray(st["type"], dtype=np.int32).tobytes())
            fh.write(st["grank"].astype(np.int32).tobytes() + st["gindex"].astype(np.int32).tobytes())


@pytest.mark.gpu
def test_shim_two_ranks_equal_library_domain_run(tmp_path):
    import domain
    import mtd
    import systems

    exe = _build(tmp_path)
    x0, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    xs = [np.ascontiguousarray(systems.wrap(systems.jitter(x0, 0.05, 61, s), L)) for s in range(3)]
    n = x0.shape[0]
    args = [str(a) for a in H.fix_args_local(pace=1)]
    probe = mtd.Metad(args, precision="mixed")
    gc = probe.ghost_cutoff
    probe.close()
    R, grid = 2, (1, 1, 2)
    dec = [domain.decompose(x, [0, 0, 0], L, grid, gc) for x in xs]
    per_rank = [[] for _ in range(R)]
    for s, ranks in enumerate(dec):
        orank = np.zeros(n, dtype=np.int64)
        opos = np.zeros(n, dtype=np.int64)
        for r, rk in enumerate(ranks):
            orank[rk["owned"]] = r
            opos[rk["owned"]] = np.arange(rk["owned"].size)
        for r, rk in enumerate(ranks):
            per_rank[r].append(dict(nlocal=rk["owned"].size, sublo=rk["lo"] + gc, subhi=rk["hi"] - gc, x=rk["x"],
                                    type=np.ones(rk["ids"].size, dtype=np.int32),
                                    grank=orank[rk["ghost"]], gindex=opos[rk["ghost"]]))
    files = []
    for r in range(R):
        files.append(str(tmp_path / ("rank%d.bin" % r)))
        _write_rank(files[-1], gc, per_rank[r])
    with open(tmp_path / "tokens.txt", "w") as fh:
        fh.write("\n".join(args) + "\n")
    subprocess.check_call([exe, "--ranks", str(R)] + files + [str(tmp_path / "tokens.txt"), str(tmp_path / "out")],
                          cwd=str(tmp_path))

    # the library's own decomposed run: one context per thread, same inputs
    red = domain.LocalAllreduce(R, timeout=120)
    ctx = [mtd.Metad(args, precision="mixed", work_dir=str(tmp_path)) for _ in range(R)]
    for r, m in enumerate(ctx):
        m.set_domain(0, r, red.for_rank(r))
    lib = [[None] * len(xs) for _ in range(R)]

    def run(r):
        try:
            for s in range(len(xs)):
                st = per_rank[r][s]
                ctx[r].set_box(st["sublo"] - gc, st["subhi"] + gc, (0, 0, 0))
                ctx[r].set_nlocal(st["nlocal"])
                f = np.zeros_like(st["x"])
                v = ctx[r].post_force(s, st["x"], f, virial=True)
                lib[r][s] = (ctx[r].compute_scalar(), ctx[r].cv, v, f)
        except BaseException:
            red.abort()
            raise

    th = [threading.Thread(target=run, args=(r,)) for r in range(R)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    for m in ctx:
        m.close()
    D = 2
    for r in range(R):
        raw = np.fromfile(str(tmp_path / ("out.%d" % r)), dtype=np.float64)
        off = 0
        for s in range(len(xs)):
            nl = per_rank[r][s]["nlocal"]
            bias, cv, v6 = raw[off], raw[off + 1:off + 1 + D], raw[off + 1 + D:off + 7 + D]
            fs = raw[off + 7 + D:off + 7 + D + 3 * nl].reshape(nl, 3)
            off += 7 + D + 3 * nl
            b_lib, cv_lib, v_lib, _ = lib[r][s]
            assert bias == b_lib and np.array_equal(cv, cv_lib) and np.array_equal(v6, v_lib)
            ftot = domain.reverse_sum(n, dec[s], [lib[q][s][3] for q in range(R)])
            want = ftot[dec[s][r]["owned"]]
            assert np.max(np.abs(fs - want)) <= 1e-13 * np.max(np.abs(want))
        assert off == raw.size
