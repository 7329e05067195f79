"""Per-atom dCV/dx export (`compute metad/atom` with `dcvdx_x/y/z`,
src/core/compute_MetaDToy.cu:79-145 through FixMetadynamics::extract,
src/core/fix_crystallize.cu:592-613) against the oracle's exact gradients.

The export is the full gradient of the CV the first SYMBOL on a CAL selects
(every neighbour term included), in caller atom order.  FP64 mode: 1e-9
relative to the largest component; mixed mode: 2e-3.
"""
import numpy as np
import pytest

import helpers as H
import oracle as O
import systems

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-9, "mixed": 2e-3}


def _grad(m, cal, n):
    return np.stack([m.extract("%s.dcvdx_%s" % (cal, a), n) for a in "xyz"], axis=1)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dcvdx_steinh_q(precision):
    x, L = systems.config1()
    x = systems.jitter(x, 0.15, 11, 0)
    m, _ = H.run_gpu(H.fix_args_q(), x, L, [(0, x)], precision=precision)
    o = O.steinh_q(6, x, L, 3.9, 18)
    g = _grad(m, "Q6", x.shape[0])
    assert H.rel(g, o["grad"]) < TOL[precision]
    # the force of the step is -dV/ds * dCV/dx: the export does not disturb it
    f = np.zeros_like(x)
    m.post_force(1, x, f)
    g2 = _grad(m, "Q6", x.shape[0])
    assert np.array_equal(g, g2)
    m.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_dcvdx_local_ql_grid(precision):
    x, L = systems.small_slab(nxy=6, nz_fcc=3, nz_bcc=4, n_liq=300)
    x = systems.jitter(x, 0.05, 3)
    m, _ = H.run_gpu(H.fix_args_local(), x, L, [(0, x), (10, x)], precision=precision)
    n = x.shape[0]
    for l in (4, 6):
        o = H.oracle_local(x, L, l)
        assert H.rel(_grad(m, "Q%d" % l, n), o["grad"]) < TOL[precision]
    m.close()


def test_dcvdx_hill_list_cvs():
    """CV_dim 4 (hill-list bias): MEAN_SOLID, the FERMI-switched FRAC and the
    k-vector S(k), each from its own symbol."""
    from test_gpu_cv4 import _args, _oracle_cvs, _system

    x, L = _system()
    m, _ = H.run_gpu(_args(), x, L, [(0, x), (1, x)], precision="fp64")
    ref = _oracle_cvs(x, L)
    n = x.shape[0]
    for cal, o in zip(["Q4", "Q6", "Q6B", "SK"], ref):
        assert H.rel(_grad(m, cal, n), o["grad"]) < 1e-9, cal
    m.close()


def test_dcvdx_unknown_cal_is_an_error():
    x, L = systems.config1()
    m, _ = H.run_gpu(H.fix_args_q(), x, L, [(0, x)], precision="fp64")
    with pytest.raises(RuntimeError, match="no SYMBOL uses CAL"):
        m.extract("Q4.dcvdx_x", x.shape[0])
    m.close()
