// neigh_body.cuh -- per-thread bodies of the cell-list and neighbour-search
// passes (one virtual block `bid` of blockDim.x atoms each), shared by their
// kernels in neigh.cu and by the persistent multi-walker step kernel.
#pragma once

#include "filter.cuh"

namespace mtd {

__device__ __forceinline__ int cell_coord(double v, const CellGrid &g, int c, double &w) {
    w = v - g.lo[c];
    if (g.periodic[c]) {
        w = w - g.L[c] * floor(w * g.invL[c]);
        if (w >= g.L[c]) w -= g.L[c];
        if (w < 0.0) w = 0.0;
    }
    int k = (int)(w * g.inv_h[c]);
    if (k < 0) k = 0;
    if (k >= g.nc[c]) k = g.nc[c] - 1;
    return k;
}

__device__ __forceinline__ void bin_body(const CellGrid &g, const SysDev &s, int bid) {
    const int i = bid * blockDim.x + threadIdx.x;
    if (i >= s.n) return;
    double w;
    const double x0 = s.x[3 * i + 0], x1 = s.x[3 * i + 1], x2 = s.x[3 * i + 2];
    // a non-finite coordinate is binned into a valid cell (cell_coord clamps),
    // matches no neighbour test (every comparison with NaN is false), and
    // fails the step: no deposit, no bias force, an error on the host
    if (!(isfinite(x0) && isfinite(x1) && isfinite(x2)) && s.status) atomicOr(&s.status->bad_pos, 1u);
    const int cx = cell_coord(x0, g, 0, w);
    const int cy = cell_coord(x1, g, 1, w);
    const int cz = cell_coord(x2, g, 2, w);
    const int cell = cell_key(g, cx, cy, cz);
    s.cellof[i] = cell;
    s.slot[i] = atomicAdd(&s.count[cell], 1);
}

// Also zeroes the cell counts for the next build (the scan has consumed them).
__device__ __forceinline__ void scatter_body(const SysDev &s, int ncell, int bid, int nblocks) {
    const int i = bid * blockDim.x + threadIdx.x;
    for (int c = i; c < ncell; c += nblocks * blockDim.x) s.count[c] = 0;
    if (i >= s.n) return;
    s.arrival[s.start[s.cellof[i]] + s.slot[i]] = i;
}

// One thread per sorted slot: the atom that arrived there takes the place of
// its rank by caller index among its cell's members (removes the atomic
// arrival order), and its sorted per-atom arrays are written there.
__device__ __forceinline__ void place_body(const CellGrid &g, const SysDev &s, int bid) {
    const int k = bid * blockDim.x + threadIdx.x;
    if (k >= s.n) return;
    const int i = s.arrival[k];
    const int c = s.cellof[i];
    const int b = s.start[c], e = s.start[c + 1];
    int rank = 0;
    for (int t = b; t < e; ++t) rank += s.arrival[t] < i;
    const int d = b + rank;
    s.perm[d] = i;
    if (s.iperm) s.iperm[i] = d;
    const double x0 = s.x[3 * i], x1 = s.x[3 * i + 1], x2 = s.x[3 * i + 2];
    s.xs[3 * d] = x0;
    s.xs[3 * d + 1] = x1;
    s.xs[3 * d + 2] = x2;
    if (s.xref) {   // skin lists: positions of this build, for the displacement test
        s.xref[3 * d] = x0;
        s.xref[3 * d + 1] = x1;
        s.xref[3 * d + 2] = x2;
    }
    // the cell coordinates bin_body keyed this atom by (same operations)
    double w0, w1, w2;
    const int cx = cell_coord(x0, g, 0, w0);
    const int cy = cell_coord(x1, g, 1, w1);
    const int cz = cell_coord(x2, g, 2, w2);
    float4 p;
    p.x = (float)(w0 - cx * g.h[0]);
    p.y = (float)(w1 - cy * g.h[1]);
    p.z = (float)(w2 - cz * g.h[2]);
    p.w = __int_as_float(pack_cell(cx, cy, cz));
    s.pf[d] = p;
    s.smask[d] = i < s.nown ? (s.mask ? s.mask[i] : -1) : 0;
}

// Fast path, valid when every periodic dimension has at least three cells:
// the 27 stencil cells are then distinct and the displacement to an atom of
// the cell at offset o is exactly o h + (off_j - off_k), so each cell's shift
// o h - off_k is formed once and a candidate costs one load and three adds.
template <int KIND>
__device__ __forceinline__ void neighbors_fast_body(const CellGrid &g, const SysDev &s, const NeighSpec &ns,
                                                    const NeighDev &nd, DevStatus *status, int bid) {
    const int k = bid * blockDim.x + threadIdx.x;
    if (k >= s.n) return;
    const GeoD gd = geo_d(g, s.xs);
    const float4 a = s.pf[k];
    const int w = __float_as_int(a.w);
    const int cx = w & 1023, cy = (w >> 10) & 1023, cz = w >> 20;
    const int nx = g.nc[0], ny = g.nc[1], nz = g.nc[2];
    int cnt = 0;
#pragma unroll 1
    for (int ox = -1; ox <= 1; ++ox) {
        int x = cx + ox;
        if (x < 0 || x >= nx) {
            if (!g.periodic[0]) continue;
            x += x < 0 ? nx : -nx;
        }
        const float sx = (float)ox * g.hf[0] - a.x;
#pragma unroll 1
        for (int oy = -1; oy <= 1; ++oy) {
            int y = cy + oy;
            if (y < 0 || y >= ny) {
                if (!g.periodic[1]) continue;
                y += y < 0 ? ny : -ny;
            }
            const float sy = (float)oy * g.hf[1] - a.y;
#pragma unroll
            for (int oz = -1; oz <= 1; ++oz) {
                int z = cz + oz;
                if (z < 0 || z >= nz) {
                    if (!g.periodic[2]) continue;
                    z += z < 0 ? nz : -nz;
                }
                const float sz = (float)oz * g.hf[2] - a.z;
                const int key = cell_key(g, x, y, z);
                const int jb = __ldg(s.start + key), je = __ldg(s.start + key + 1);
                float4 nxt = jb < je ? __ldg(s.pf + jb) : make_float4(0.f, 0.f, 0.f, 0.f);
                for (int j = jb; j < je; ++j) {
                    const float4 b = nxt;
                    if (j + 1 < je) nxt = __ldg(s.pf + j + 1);
                    const float dx = b.x + sx, dy = b.y + sy, dz = b.z + sz;
                    const float r2f = dx * dx + dy * dy + dz * dz;
                    if (r2f > ns.hi2 || j == k) continue;
                    bool in;
                    if (KIND == NK_CAND || (KIND != NK_SWITCH && r2f < ns.lo2 && r2f > 1e-6f)) {
                        in = true;
                    } else {
                        in = exact_decide<KIND>(exact_spec(gd, ns), s.xs, k, j);
                    }
                    if (!in) continue;
                    if (cnt < nd.M) nd.list[(size_t)cnt * s.npad + k] = j;
                    ++cnt;
                }
            }
        }
    }
    nd.count[k] = cnt;
    if (cnt > nd.M) atomicMax(KIND == NK_CAND ? &status->cand_overflow : &status->overflow, (unsigned)cnt);
}

}  // namespace mtd
