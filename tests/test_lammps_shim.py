"""The LAMMPS shim (metad-toy_b200/lammps: fix metad, compute metad/atom and
the plugin registration) against stand-in LAMMPS classes (tests/lammps_stub):
it compiles against the API it uses, and driven like LAMMPS drives a fix
(plugin load, fix and compute from deck tokens, init, post_force with the
virial flag each step) it gives exactly the library's own step: same forces
bit for bit, bias, CVs, virial and per-atom exports."""
import os
import struct
import subprocess

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
        "-L" + PKG, "-lmetad_b200", "-Wl,-rpath," + PKG, "-o", exe]
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
