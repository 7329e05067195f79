"""mtd_sk_noalloc: the allocation-free k-vector structure factor, checked
through the C ABI against a context's STRU_FACTOR_K unit (mtd_post_force) on
the same atoms and k-vectors, on two calls in a row.

Tolerances (relative): FP64 1e-10, mixed 1e-5 on S; rho against a NumPy FP64
sum 1e-10 (FP64) and 1e-4 of max |rho| (mixed).  The two paths differ only in
the number of partial-sum blocks, i.e. in the order of the FP64 sums.
"""
import numpy as np
import pytest

import helpers as H
import mtd
import systems


def _system(seed):
    x = systems.lattice(6, 6, 6, 3.615, systems.FCC_BASIS)
    L = np.array([6 * 3.615] * 3)
    return systems.wrap(systems.jitter(x, 0.15, seed), L), L


def _context_s(x, L, nk, kmag, seed, precision, groups=None, mask=None):
    group = "all" if groups is None else "half"
    args = ["GAUSSIAN", 0.5, 0.005, 10.0, "PACE", 10,
            "CAL", "NAME", "SK", "STRU_FACTOR_K", group, "nk", nk, "kmag", kmag, "seed", seed,
            "SYMBOL", "v1", "SK.AVE", "CV_dim", 1, "DIM", 1, 0.0, 1000.0, 500, "v1", "WT", 0]
    m, out = H.run_gpu(args, x, L, [(1, x)], precision=precision, groups=groups, mask=mask)
    return out[0][0][0]


def test_rejects_bad_sizes_without_touching_the_device():
    with pytest.raises(mtd.MetadError, match=r"nk must be in \[1, 1024\]"):
        mtd.sk_noalloc(10, 0, 0, 0, 0)
    with pytest.raises(mtd.MetadError, match=r"nk must be in \[1, 1024\]"):
        mtd.sk_noalloc(10, 0, 0, 1025, 0)
    with pytest.raises(mtd.MetadError, match="n must be >= 0"):
        mtd.sk_noalloc(-1, 0, 0, 4, 0)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_matches_context_on_two_calls_in_a_row(precision):
    import torch

    nk, kmag, seed = 48, systems.KMAG_111, 5
    kv = systems.kvectors(nk, kmag, seed)
    d_k = torch.tensor(kv, dtype=torch.float64, device="cuda")
    d_s = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_rho = torch.zeros(2 * nk, dtype=torch.float64, device="cuda")
    tol_s = 1e-10 if precision == "fp64" else 1e-5
    tol_rho = 1e-10 if precision == "fp64" else 1e-4
    first = None
    for call, xseed in enumerate([3, 4]):
        x, L = _system(xseed)
        d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
        mtd.sk_noalloc(x.shape[0], d_x.data_ptr(), d_k.data_ptr(), nk, d_s.data_ptr(), rho_ptr=d_rho.data_ptr(),
                       precision=precision)
        torch.cuda.synchronize()
        s = float(d_s.item())
        ref = _context_s(x, L, nk, kmag, seed, precision)
        assert H.rel(s, ref) < tol_s
        ph = x @ kv.T
        rho = np.stack([np.cos(ph).sum(0), np.sin(ph).sum(0)], axis=1).reshape(-1)
        assert H.rel(d_rho.cpu().numpy(), rho) < tol_rho
        if call == 0:
            first = (x, s)
    # the scratch holds the second call's partials now; a repeat of the first
    # input must give the first result exactly
    x, s = first
    d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
    mtd.sk_noalloc(x.shape[0], d_x.data_ptr(), d_k.data_ptr(), nk, d_s.data_ptr(), precision=precision)
    torch.cuda.synchronize()
    assert float(d_s.item()) == s


@pytest.mark.gpu
def test_group_mask_matches_context():
    import torch

    nk, kmag, seed = 16, systems.KMAG_111, 11
    x, L = _system(8)
    mask = np.where(np.arange(x.shape[0]) % 2 == 0, 1 | 2, 1).astype(np.int32)
    kv = systems.kvectors(nk, kmag, seed)
    d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
    d_m = torch.tensor(mask, dtype=torch.int32, device="cuda")
    d_k = torch.tensor(kv, dtype=torch.float64, device="cuda")
    d_s = torch.zeros(1, dtype=torch.float64, device="cuda")
    mtd.sk_noalloc(x.shape[0], d_x.data_ptr(), d_k.data_ptr(), nk, d_s.data_ptr(), mask_ptr=d_m.data_ptr(),
                   groupbit=2, precision="fp64")
    torch.cuda.synchronize()
    ref = _context_s(x, L, nk, kmag, seed, "fp64", groups={"all": 1, "half": 2}, mask=mask)
    assert H.rel(float(d_s.item()), ref) < 1e-10


@pytest.mark.gpu
def test_largest_k_set_and_empty_input():
    """nk = 1024, the stated maximum (63 partial blocks fill the fixed
    scratch), against a NumPy FP64 sum; then n = 0, which gives S = 0 and
    rho = 0 without reading any atom."""
    import torch

    nk = 1024
    x, L = _system(21)
    kv = systems.kvectors(nk, systems.KMAG_111, 17)
    d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
    d_k = torch.tensor(kv, dtype=torch.float64, device="cuda")
    d_s = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_rho = torch.zeros(2 * nk, dtype=torch.float64, device="cuda")
    mtd.sk_noalloc(x.shape[0], d_x.data_ptr(), d_k.data_ptr(), nk, d_s.data_ptr(), rho_ptr=d_rho.data_ptr(),
                   precision="fp64")
    torch.cuda.synchronize()
    ph = x @ kv.T
    re, im = np.cos(ph).sum(0), np.sin(ph).sum(0)
    assert H.rel(d_rho.cpu().numpy(), np.stack([re, im], axis=1).reshape(-1)) < 1e-10
    assert H.rel(float(d_s.item()), float(np.sum(re * re + im * im)) / x.shape[0] / nk) < 1e-10
    d_s.fill_(7.0)
    d_rho.fill_(7.0)
    mtd.sk_noalloc(0, 0, d_k.data_ptr(), nk, d_s.data_ptr(), rho_ptr=d_rho.data_ptr(), precision="fp64")
    torch.cuda.synchronize()
    assert float(d_s.item()) == 0.0 and np.all(d_rho.cpu().numpy() == 0.0)


@pytest.mark.gpu
def test_a_call_allocates_no_device_memory():
    """After the set-up call, further calls leave the device's free memory
    unchanged (cudaMemGetInfo before and after): the scratch is the static
    array, not memory from an allocator."""
    import torch

    nk = 96
    x, L = _system(22)
    kv = systems.kvectors(nk, systems.KMAG_111, 23)
    d_x = torch.tensor(x, dtype=torch.float64, device="cuda")
    d_k = torch.tensor(kv, dtype=torch.float64, device="cuda")
    d_s = torch.zeros(1, dtype=torch.float64, device="cuda")
    d_rho = torch.zeros(2 * nk, dtype=torch.float64, device="cuda")
    for precision in ("mixed", "fp64"):
        mtd.sk_noalloc(x.shape[0], d_x.data_ptr(), d_k.data_ptr(), nk, d_s.data_ptr(), rho_ptr=d_rho.data_ptr(),
                       precision=precision)   # set-up and first launch of each kernel
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for precision in ("mixed", "fp64", "mixed"):
        mtd.sk_noalloc(x.shape[0], d_x.data_ptr(), d_k.data_ptr(), nk, d_s.data_ptr(), rho_ptr=d_rho.data_ptr(),
                       precision=precision)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
