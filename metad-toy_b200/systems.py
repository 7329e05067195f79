"""Seeded synthetic atom configurations for the metadynamics hot path.

The reference measures on LAMMPS decks, not on a public dataset; these
generators build the same kinds of systems (FCC/BCC lattices, a hard-core
liquid, jittered lattices) deterministically from a seed, so the GPU path,
the CPU oracle and the benchmark see identical positions.

Positions are float64 arrays of shape (n, 3) inside [0, L) on periodic boxes.
"""
from __future__ import annotations

import math

import numpy as np

FCC_BASIS = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)
BCC_BASIS = np.array([[0, 0, 0], [0.5, 0.5, 0.5]], dtype=np.float64)


def lattice(nx, ny, nz, a, basis, origin=(0.0, 0.0, 0.0)):
    """Cells ordered x-slowest; `a` is a scalar or (ax, ay, az)."""
    a = np.broadcast_to(np.asarray(a, dtype=np.float64), (3,))
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 1, 3)
    x = ((g + basis[None]) * a).reshape(-1, 3)
    return x + np.asarray(origin, dtype=np.float64)


def fcc(nc, a):
    return lattice(nc, nc, nc, a, FCC_BASIS)


def bcc(nc, a):
    return lattice(nc, nc, nc, a, BCC_BASIS)


def wrap(x, L):
    L = np.asarray(L, dtype=np.float64)
    return x - L * np.floor(x / L)


def jitter(x, sigma, seed, step=0):
    """x + N(0, sigma) per component from a Philox stream keyed by (seed, step)."""
    rng = np.random.Generator(np.random.Philox(key=int(seed), counter=[0, 0, 0, int(step)]))
    return x + rng.normal(0.0, sigma, size=x.shape)


def splitmix64(seed):
    s = seed & 0xFFFFFFFFFFFFFFFF
    while True:
        s = (s + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        yield z ^ (z >> 31)


def kvectors(nk, kmag, seed):
    """Directions uniform on the sphere (Marsaglia 1972) from SplitMix64(seed);
    the same sequence the library's STRU_FACTOR_K builds from `seed`."""
    g = splitmix64(seed)

    def uni():
        return (next(g) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0

    out = np.zeros((nk, 3))
    for q in range(nk):
        while True:
            a, b = uni(), uni()
            r2 = a * a + b * b
            if 0.0 < r2 < 1.0:
                break
        t = 2.0 * math.sqrt(1.0 - r2)
        out[q] = (kmag * a * t, kmag * b * t, kmag * (1.0 - 2.0 * r2))
    return out


def hardcore_liquid(n, lo, hi, L, rmin, seed, fixed=None, batch=4096):
    """Random sequential addition of n points in the slab lo <= z < hi of a periodic
    box L with pairwise distance >= rmin, also from the points in `fixed`."""
    from scipy.spatial import cKDTree

    rng = np.random.Generator(np.random.Philox(key=int(seed)))
    acc = np.zeros((0, 3))
    box = np.asarray(L, dtype=np.float64)
    fixed = np.zeros((0, 3)) if fixed is None else fixed
    if fixed.shape[0]:
        # only crystal atoms within rmin of the slab can block an insertion
        t = wrap(fixed[:, 2] - lo, box[2])
        fixed = fixed[(t < hi - lo + rmin) | (t > box[2] - rmin)]
    ftree = cKDTree(wrap(fixed, box), boxsize=box) if fixed.shape[0] else None
    rate = 0.5
    for _ in range(100000):
        need = n - acc.shape[0]
        if need <= 0:
            break
        size = int(min(max(batch, 2 * need / max(rate, 1e-3)), 1 << 18))
        cand = rng.random((size, 3)) * np.array([box[0], box[1], hi - lo]) + np.array([0.0, 0.0, lo])
        cand = wrap(cand, box)
        keep = np.ones(size, bool)
        if ftree is not None:
            keep &= ftree.query(cand, k=1, distance_upper_bound=rmin)[0] >= rmin
        if acc.shape[0]:
            atree = cKDTree(acc, boxsize=box)
            keep &= atree.query(cand, k=1, distance_upper_bound=rmin)[0] >= rmin
        cand = cand[keep]
        if cand.shape[0]:
            # among this batch's survivors the later member of a close pair is dropped
            pairs = cKDTree(cand, boxsize=box).query_pairs(rmin, output_type="ndarray")
            drop = np.zeros(cand.shape[0], bool)
            if pairs.shape[0]:
                drop[np.maximum(pairs[:, 0], pairs[:, 1])] = True
            cand = cand[~drop]
        rate = max(cand.shape[0] / size, 1e-3)
        acc = np.concatenate([acc, cand[:need]])
    else:
        raise RuntimeError("hard-core insertion did not converge")
    return acc


def config1(seed=2024):
    """4,000 atoms: 10x10x10 FCC, a = 5.26 A, periodic 52.6 A box."""
    a, nc = 5.26, 10
    return fcc(nc, a), np.array([nc * a] * 3)


def config2(seed=2024, n_fcc_z=36, n_bcc_z=47, n_total=256000, rho_liq=0.021, rmin=3.0, gap=1.0):
    """256,000 atoms in z-stacked slabs on a 125.4 x 125.4 A cross-section:
    FCC 24x24x36 cells = 82,944 atoms (a_xy 5.225, a_z 5.26), BCC 30x30x47
    cells = 84,600 atoms (a 4.18), hard-core liquid (0.021 A^-3, 3.0 A core,
    also against the crystal) for the remaining 88,456; `gap` A of extra
    spacing separates the FCC and BCC slabs."""
    Lxy = 30 * 4.18
    a_fcc_z = 5.26
    fcc_x = lattice(24, 24, n_fcc_z, (Lxy / 24, Lxy / 24, a_fcc_z), FCC_BASIS)
    z0 = n_fcc_z * a_fcc_z + gap
    bcc_x = lattice(30, 30, n_bcc_z, 4.18, BCC_BASIS, origin=(0.0, 0.0, z0))
    z1 = z0 + n_bcc_z * 4.18
    n_liq = n_total - fcc_x.shape[0] - bcc_x.shape[0]
    thick = n_liq / (rho_liq * Lxy * Lxy)
    L = np.array([Lxy, Lxy, z1 + thick])
    crystal = np.concatenate([fcc_x, bcc_x])
    liq = hardcore_liquid(n_liq, z1, z1 + thick, L, rmin, seed, fixed=crystal)
    x = wrap(np.concatenate([crystal, liq]), L)
    return x, L


def config3(seed=2024, nc=64, a=5.26, sigma=0.2):
    """64^3 FCC cells = 1,048,576 atoms, a = 5.26 A, jitter N(0, 0.2 A)."""
    x = jitter(fcc(nc, a), sigma, seed)
    return x, np.array([nc * a] * 3)


KMAG_111 = 2.0 * math.pi * math.sqrt(3.0) / 5.26


def small_slab(seed=7, nxy=5, nz_fcc=2, nz_bcc=3, n_liq=200):
    """A few-thousand-atom analogue of config2 for parity tests."""
    a_bcc = 4.18
    Lxy = nxy * a_bcc * 1.0
    fcc_x = lattice(4, 4, nz_fcc, (Lxy / 4, Lxy / 4, 5.26), FCC_BASIS)
    z0 = nz_fcc * 5.26
    bcc_x = lattice(nxy, nxy, nz_bcc, a_bcc, BCC_BASIS, origin=(0, 0, z0))
    z1 = z0 + nz_bcc * a_bcc
    thick = n_liq / (0.021 * Lxy * Lxy)
    L = np.array([Lxy, Lxy, z1 + thick])
    crystal = np.concatenate([fcc_x, bcc_x])
    liq = hardcore_liquid(n_liq, z1, z1 + thick, L, 3.0, seed, fixed=crystal)
    return wrap(np.concatenate([crystal, liq]), L), L


CV4_LO = np.array([0.20, 0.35, 0.0, 0.05])
CV4_HI = np.array([0.45, 0.60, 1.0, 0.35])


def cv4_hills(n=20000, seed=5, sigma=0.02, height=0.005):
    """Hill centres of a seeded 4D CV trajectory (Q4.AVE, Q6.AVE, local-Q6
    fraction, S(k)): an Ornstein-Uhlenbeck walk reflected into CV4_LO..CV4_HI,
    one hill per PACE, steps of 0.35 sigma per dimension."""
    rng = np.random.default_rng(seed)
    span = CV4_HI - CV4_LO
    x = CV4_LO + 0.5 * span
    c = np.zeros((n, 4))
    for i in range(n):
        x = x + 0.35 * sigma * rng.standard_normal(4) - 0.002 * (x - (CV4_LO + 0.5 * span))
        x = np.where(x < CV4_LO, 2 * CV4_LO - x, x)
        x = np.where(x > CV4_HI, 2 * CV4_HI - x, x)
        c[i] = x
    return c, np.full(n, height), np.full(n, sigma)


def walker_system(n, seed, a=5.26, nxy=6, rho_liq=0.021, jitter_liq=0.4, gap=1.0):
    """n atoms: an FCC slab (nxy x nxy cells, a) holding about half of them and a
    disordered slab at rho_liq (a simple-cubic lattice at that density with
    N(0, jitter_liq) displacements) holding the rest, periodic box."""
    rng = np.random.default_rng(seed)
    Lxy = nxy * a
    per_layer = 4 * nxy * nxy
    nz = max(1, int(round(0.5 * n / per_layer)))
    while nz > 1 and nz * per_layer > n - 64:
        nz -= 1
    crystal = lattice(nxy, nxy, nz, a, FCC_BASIS)
    n_liq = n - crystal.shape[0]
    z0 = nz * a + gap
    spacing = (1.0 / rho_liq) ** (1.0 / 3.0)
    m = max(1, int(round(Lxy / spacing)))
    d = Lxy / m
    nzl = int(math.ceil(n_liq / (m * m)))
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(nzl), indexing="ij"), -1).reshape(-1, 3)
    g = g[np.lexsort((g[:, 0], g[:, 1], g[:, 2]))][:n_liq]
    liq = (g + 0.5) * np.array([d, d, d]) + np.array([0.0, 0.0, z0]) + rng.normal(0.0, jitter_liq, (n_liq, 3))
    L = np.array([Lxy, Lxy, z0 + nzl * d + gap])
    return wrap(np.concatenate([crystal, liq]), L), L
