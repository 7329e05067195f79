// neigh.cu -- cell list and neighbour lists on the device.
//
// Replaces the host CSR flatten of LAMMPS neighbour lists plus the selection
// kernels get_environment_Steinhardt_Q (src/cvs/CVs_Steinhardt.cu:1324-1406),
// get_environment_Steinhardt_LocalQ (src/cvs/CVs_Steinhardt_Local.cu:1210-1285)
// and get_environment_Strufactor (src/cvs/CVs_Strufactor.cu:1014-1080).
//
// Per step: bin atoms to cells (counting sort: histogram, scan, scatter in
// atomic arrival order, then every atom moves to its rank by caller index
// within its cell, so the order is deterministic), then
// one thread per sorted atom walks its 9 neighbour-cell columns (z-adjacent
// cells are contiguous in the sorted order).  A candidate is decided by its
// FP32 cell-relative distance unless it lies within ~1e-5 of the bound, where
// the FP64 test on the caller's raw coordinates (the FP64 oracle's operation
// order) decides -- the neighbour sets are exact.
//
// With skin lists (NEIGH_SKIN) the cell list and candidate lists (cutoff +
// skin) are rebuilt only when k_refresh finds an atom that moved more than
// skin / 2 since the last rebuild (or NEIGH_EVERY steps have passed); every
// step the candidates are filtered to the exact lists at the current
// positions, so the neighbour sets are exact either way.  This is the model
// of the reference, which reads LAMMPS's skin lists and filters them by
// r < cutoff_r every step (src/cvs/CVs_Steinhardt.cu:135-147,
// src/core/neigh_hub.cu:191-222).
#include "persist.cuh"

#include <math_constants.h>

namespace mtd {

namespace {


// The rebuild kernels return at once while the skin gate is closed (the
// gate is written by k_refresh, complete before pdl_entry returns).
__device__ __forceinline__ bool gate_closed(const SkinState *sk) {
    return sk && *(volatile const unsigned *)&sk->gate == 0u;
}


__global__ void k_bin(CellGrid g, SysDev s) {
    pdl_entry();
    if (gate_closed(s.skin)) return;
    bin_body(g, s, blockIdx.x);
}

// Exclusive block scan of one value per thread (blockDim.x == kScanBlock).
constexpr int kScanBlock = 1024;
__device__ __forceinline__ int block_excl_scan(int v, int &total) {
    __shared__ int warp_tot[32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int t = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[31];
    const int excl = (warp > 0 ? warp_tot[warp - 1] : 0) + x - v;
    __syncthreads();
    return excl;
}

// Three-pass exclusive scan of the cell histogram: per-block scan, scan of the
// block totals, add-back.  The totals live in start[ncell + 1 ...].
__global__ void __launch_bounds__(kScanBlock) k_scan_blocks(const int *__restrict__ count, int *__restrict__ start,
                                                            int *__restrict__ bsum, int ncell, const SkinState *skin) {
    pdl_entry();
    if (gate_closed(skin)) return;
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    int total;
    const int e = block_excl_scan(i < ncell ? count[i] : 0, total);
    if (i < ncell) start[i] = e;
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_top(int *__restrict__ bsum, int nb, int *__restrict__ start,
                                                         int ncell, const SkinState *skin) {
    pdl_entry();
    if (gate_closed(skin)) return;
    int carry = 0;
    for (int base = 0; base < nb; base += kScanBlock) {
        const int i = base + threadIdx.x;
        int total;
        const int e = block_excl_scan(i < nb ? bsum[i] : 0, total);
        if (i < nb) bsum[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) start[ncell] = carry;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_add(int *__restrict__ start, const int *__restrict__ bsum,
                                                         int ncell, const SkinState *skin) {
    pdl_entry();
    if (gate_closed(skin)) return;
    const int i = blockIdx.x * kScanBlock + threadIdx.x;
    if (i < ncell) start[i] += bsum[blockIdx.x];
}

// Single-kernel add-back when the block totals fit one block: each block sums
// the totals of the blocks before it (the last block also writes the total).
__global__ void __launch_bounds__(kScanBlock) k_scan_add_fused(int *__restrict__ start, const int *__restrict__ bsum,
                                                               int ncell, int nb, const SkinState *skin) {
    pdl_entry();
    if (gate_closed(skin)) return;
    __shared__ int red[32];
    const int b = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int v = threadIdx.x < b ? bsum[threadIdx.x] : 0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    int off = 0;
#pragma unroll 1
    for (int w = 0; w < (kScanBlock >> 5); ++w) off += red[w];
    const int i = b * kScanBlock + threadIdx.x;
    if (i < ncell) start[i] += off;
    if (b == nb - 1 && threadIdx.x == 0) start[ncell] = off + bsum[b];
}



// Also zeroes the cell counts for the next build (the scan has consumed them).
__global__ void k_scatter(SysDev s, int ncell) {
    pdl_entry();
    if (gate_closed(s.skin)) return;
    scatter_body(s, ncell, blockIdx.x, gridDim.x);
}

// One thread per sorted slot: the atom that arrived there takes the place of
// its rank by caller index among its cell's members (removes the atomic
// arrival order), and its sorted per-atom arrays are written there.
__global__ void k_place(CellGrid g, SysDev s) {
    pdl_entry();
    if (gate_closed(s.skin)) return;
    place_body(g, s, blockIdx.x);
}

template <int KIND>
__global__ void __launch_bounds__(kBlock) k_neighbors(CellGrid g, SysDev s, NeighSpec ns, NeighDev nd,
                                                      DevStatus *status) {
    pdl_entry();
    if (gate_closed(s.skin)) return;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= s.n) return;
    const GeoF gf = geo_f(g, s.pf);
    const GeoD gd = geo_d(g, s.xs);
    const float4 a = s.pf[k];
    const int w = __float_as_int(a.w);
    const int cx = w & 1023, cy = (w >> 10) & 1023, cz = w >> 20;
    const int nz = g.nc[2];
    int cnt = 0;
    for (int ox = -1; ox <= 1; ++ox) {
        int x = cx + ox;
        if (g.periodic[0]) {
            if (g.nc[0] < 3 && ox != 0 && (g.nc[0] == 1 || ox == -1)) continue;
            x = (x + g.nc[0]) % g.nc[0];
        } else if (x < 0 || x >= g.nc[0]) continue;
        for (int oy = -1; oy <= 1; ++oy) {
            int y = cy + oy;
            if (g.periodic[1]) {
                if (g.nc[1] < 3 && oy != 0 && (g.nc[1] == 1 || oy == -1)) continue;
                y = (y + g.nc[1]) % g.nc[1];
            } else if (y < 0 || y >= g.nc[1]) continue;
            const int col = (x * g.nc[1] + y) * nz;
            // z cells of the column: one contiguous range unless the stencil wraps
            int zr[3][2], nr = 0;
            if (nz >= 3 && cz >= 1 && cz <= nz - 2) {
                zr[0][0] = cz - 1;
                zr[0][1] = cz + 1;
                nr = 1;
            } else if (nz >= 3 && g.periodic[2]) {
                if (cz == 0) {
                    zr[0][0] = 0; zr[0][1] = 1; zr[1][0] = nz - 1; zr[1][1] = nz - 1; nr = 2;
                } else {
                    zr[0][0] = nz - 2; zr[0][1] = nz - 1; zr[1][0] = 0; zr[1][1] = 0; nr = 2;
                }
            } else {
                zr[0][0] = max(cz - 1, 0);
                zr[0][1] = min(cz + 1, nz - 1);
                nr = 1;
            }
            for (int r = 0; r < nr; ++r) {
                const int jb = s.start[col + zr[r][0]], je = s.start[col + zr[r][1] + 1];
                for (int j = jb; j < je; ++j) {
                    if (j == k) continue;
                    const float4 b = s.pf[j];
                    float dx, dy, dz;
                    disp_f(gf, a, b, dx, dy, dz);
                    const float r2f = dx * dx + dy * dy + dz * dz;
                    if (r2f > ns.hi2) continue;
                    bool in;
                    if (KIND != NK_SWITCH && r2f < ns.lo2 && r2f > 1e-6f) {
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
    if (cnt > nd.M) atomicMax(&status->overflow, (unsigned)cnt);
}


// Fast path, valid when every periodic dimension has at least three cells
// (neighbors_fast_body).
template <int KIND>
__global__ void __launch_bounds__(kBlock) k_neighbors_fast(CellGrid g, SysDev s, NeighSpec ns, NeighDev nd,
                                                           DevStatus *status) {
    pdl_entry();
    if (gate_closed(s.skin)) return;
    neighbors_fast_body<KIND>(g, s, ns, nd, status, blockIdx.x);
}

// Same lists as k_neighbors_fast (same cells in the same order, same tests),
// with the warp's divergence taken out of the cell loop: each thread first
// records the non-empty cells of its 27-cell stencil in shared memory (a
// uniform pass), then walks all its candidates in one flat loop, moving to the
// next recorded cell when one runs out.  A warp then runs as many trips as
// its busiest lane has candidates, instead of, for each of 27 cells, as many
// as the fullest lane's cell holds.
constexpr int kFlatBlock = 128;
template <int KIND>
__global__ void __launch_bounds__(kFlatBlock) k_neighbors_flat(CellGrid g, SysDev s, NeighSpec ns, NeighDev nd,
                                                               DevStatus *status) {
    pdl_entry();
    // [cell][thread]: a lane's entry sits in the same bank whatever cell it reads
    __shared__ int2 rng[27][kFlatBlock];
    if (gate_closed(s.skin)) return;
    const int tid = threadIdx.x;
    const int k = blockIdx.x * blockDim.x + tid;
    if (k >= s.n) return;   // no block-wide synchronisation below
    const GeoD gd = geo_d(g, s.xs);
    const float4 a = s.pf[k];
    const int w = __float_as_int(a.w);
    const int cx = w & 1023, cy = (w >> 10) & 1023, cz = w >> 20;
    const int nx = g.nc[0], ny = g.nc[1], nz = g.nc[2];
    // the cell shift o h - offset for o = -1, 0, 1 per dimension (as k_neighbors_fast forms it)
    const float shx[3] = {-g.hf[0] - a.x, 0.f * g.hf[0] - a.x, g.hf[0] - a.x};
    const float shy[3] = {-g.hf[1] - a.y, 0.f * g.hf[1] - a.y, g.hf[1] - a.y};
    const float shz[3] = {-g.hf[2] - a.z, 0.f * g.hf[2] - a.z, g.hf[2] - a.z};
    int nr = 0;
#pragma unroll 1
    for (int ox = 0; ox < 3; ++ox) {
        int x = cx + ox - 1;
        if (x < 0 || x >= nx) {
            if (!g.periodic[0]) continue;
            x += x < 0 ? nx : -nx;
        }
#pragma unroll 1
        for (int oy = 0; oy < 3; ++oy) {
            int y = cy + oy - 1;
            if (y < 0 || y >= ny) {
                if (!g.periodic[1]) continue;
                y += y < 0 ? ny : -ny;
            }
#pragma unroll
            for (int oz = 0; oz < 3; ++oz) {
                int z = cz + oz - 1;
                if (z < 0 || z >= nz) {
                    if (!g.periodic[2]) continue;
                    z += z < 0 ? nz : -nz;
                }
                const int key = cell_key(g, x, y, z);
                const int b0 = __ldg(s.start + key), b1 = __ldg(s.start + key + 1);
                // end < 2^26, the stencil offsets (2 bits each) above it
                const unsigned code = (unsigned)ox | ((unsigned)oy << 2) | ((unsigned)oz << 4);
                if (b0 < b1) rng[nr++][tid] = make_int2(b0, (int)((unsigned)b1 | (code << 26)));
            }
        }
    }
    int cnt = 0;
    int r = 0, j = 0, je = 0;
    float sx = 0.f, sy = 0.f, sz = 0.f;
    auto open = [&]() {
        const int2 e = rng[r++][tid];
        const unsigned code = (unsigned)e.y >> 26;
        j = e.x;
        je = e.y & ((1 << 26) - 1);
        const unsigned qx = code & 3u, qy = (code >> 2) & 3u, qz = code >> 4;
        sx = qx == 0 ? shx[0] : (qx == 1 ? shx[1] : shx[2]);
        sy = qy == 0 ? shy[0] : (qy == 1 ? shy[1] : shy[2]);
        sz = qz == 0 ? shz[0] : (qz == 1 ? shz[1] : shz[2]);
    };
    bool live = nr > 0;
    float4 nxt = make_float4(0.f, 0.f, 0.f, 0.f);
    if (live) {
        open();
        nxt = __ldg(s.pf + j);
    }
    while (live) {
        const float4 b = nxt;
        const int jj = j;
        const float dx = b.x + sx, dy = b.y + sy, dz = b.z + sz;
        if (++j == je) {
            live = r < nr;
            if (live) open();
        }
        if (live) nxt = __ldg(s.pf + j);
        const float r2f = dx * dx + dy * dy + dz * dz;
        if (r2f > ns.hi2 || jj == k) continue;
        bool in;
        if (KIND == NK_CAND || (KIND != NK_SWITCH && r2f < ns.lo2 && r2f > 1e-6f)) {
            in = true;
        } else {
            in = exact_decide<KIND>(exact_spec(gd, ns), s.xs, k, jj);
        }
        if (!in) continue;
        if (cnt < nd.M) nd.list[(size_t)cnt * s.npad + k] = jj;
        ++cnt;
    }
    nd.count[k] = cnt;
    if (cnt > nd.M) atomicMax(KIND == NK_CAND ? &status->cand_overflow : &status->overflow, (unsigned)cnt);
}

constexpr int kMaxCapList = 64;

// STEINH Q cap: keep the `cap` nearest by (r2, caller index), the order of the
// reference's strict-'>' insertion with ties resolved canonically.
__global__ void __launch_bounds__(kBlock) k_select_cap(CellGrid g, SysDev s, NeighSpec ns, NeighDev nd) {
    pdl_entry();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= s.n) return;
    const GeoD gd = geo_d(g, s.xs);
    const int c = min(nd.count[k], min(nd.M, kMaxCapList));
    double r2[kMaxCapList];
    int id[kMaxCapList];
    const double xk[3] = {s.xs[3 * k], s.xs[3 * k + 1], s.xs[3 * k + 2]};
    for (int t = 0; t < c; ++t) {
        const int j = nd.list[(size_t)t * s.npad + k];
        const double xj[3] = {s.xs[3 * j], s.xs[3 * j + 1], s.xs[3 * j + 2]};
        double d[3];
        r2[t] = exact_disp(gd, xk, xj, d);
        id[t] = s.perm[j];
    }
    double kr2 = CUDART_INF;
    int kid = 0x7fffffff;
    for (int t = 0; t < c; ++t) {
        int rank = 0;
        for (int u = 0; u < c; ++u)
            if (r2[u] < r2[t] || (r2[u] == r2[t] && id[u] < id[t])) ++rank;
        if (rank < ns.cap) nd.list[(size_t)t * s.npad + k] |= (1 << kFlagBit);
        if (c > ns.cap && rank == ns.cap - 1) {
            kr2 = r2[t];
            kid = id[t];
        }
    }
    nd.key_r2[k] = kr2;
    nd.key_id[k] = kid;
    nd.nkept[k] = c < ns.cap ? c : ns.cap;
}

// Skin lists, every step: one thread per sorted slot of the last rebuild.
// Repacks the caller's positions into that order (xs, and pf as FP32 offsets
// from the slot's build cell, which stays within half a cell of it while the
// lists are valid), refreshes the group mask, and opens the gate when a
// rebuild is due: an atom moved more than skin / 2 (minimum image) since the
// build, a non-finite position, NEIGH_EVERY reached, or force (the sorted
// order is not valid yet, or the last rebuild gave up: nothing else is read).
__global__ void k_refresh(CellGrid g, SysDev s, int every, double half2, int force) {
    pdl_entry();
    SkinState *sk = s.skin;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    // a rebuild that gave up leaves the sorted order and lists unusable: rebuild as if forced
    if (*(volatile const unsigned *)&sk->invalid) force = 1;
    if (k == 0 && (force || (every > 0 && sk->age >= (unsigned)every))) atomicOr(&sk->gate, 1u);
    if (force || k >= s.n) return;
    const int i = s.perm[k];
    const double x[3] = {s.x[3 * (size_t)i], s.x[3 * (size_t)i + 1], s.x[3 * (size_t)i + 2]};
    const bool finite = isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]);
    if (!finite && s.status) atomicOr(&s.status->bad_pos, 1u);
    double d2 = 0.0;
    const float4 p = s.pf[k];
    const int w = __float_as_int(p.w);
    const int cc[3] = {w & 1023, (w >> 10) & 1023, w >> 20};
    float off[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double t = x[c] - s.xref[3 * (size_t)k + c];
        double o = (x[c] - g.lo[c]) - cc[c] * g.h[c];
        if (g.periodic[c]) {
            t -= g.L[c] * rint(t * g.invL[c]);
            o -= g.L[c] * rint((o - 0.5 * g.h[c]) * g.invL[c]);
        }
        d2 += t * t;
        off[c] = (float)o;
    }
    const unsigned moved = !(finite && d2 <= half2);
    const unsigned ballot = __ballot_sync(__activemask(), moved);   // one atomic per warp
    if (ballot && (threadIdx.x & 31) == __ffs(ballot) - 1) atomicOr(&sk->gate, 1u);
    s.xs[3 * (size_t)k] = x[0];
    s.xs[3 * (size_t)k + 1] = x[1];
    s.xs[3 * (size_t)k + 2] = x[2];
    s.pf[k] = make_float4(off[0], off[1], off[2], p.w);
    s.smask[k] = i < s.nown ? (s.mask ? s.mask[i] : -1) : 0;
}

// Skin lists, every step: the exact lists of one environment from its
// candidates.  reset (the first kernel after the gated rebuild kernels)
// records the step in the skin state and closes the gate.
template <int KIND>
__global__ void __launch_bounds__(kBlock) k_filter(CellGrid g, SysDev s, NeighSpec ns, NeighDev nd, NeighDev cand,
                                                   DevStatus *status, SkinState *reset) {
    pdl_entry();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (reset && k == 0) {
        if (reset->gate) {
            reset->age = 1;
            reset->builds += 1;
        } else {
            reset->age += 1;
        }
        reset->gate = 0;
    }
    if (k >= s.n) return;
    filter_atom<KIND>(geo_f(g, s.pf), geo_d(g, s.xs), s.xs, ns, cand, nd, s.npad, k, status);
}

// Skin lists, the whole rebuild as one cooperative launch: while the gate is
// closed every block returns at once (one launch instead of six that each
// return at once); when it is open the phases run with grid barriers between
// them: cell counts zeroed, bin, chunk scan, chunk offsets, scatter, place,
// candidates.  The same per-thread bodies and 256-atom blocks as the separate
// kernels, so the sorted order and the candidate lists are the same.  A
// barrier wait that runs out marks the step (status->timeout, no deposit, no
// bias force) and the skin state invalid (the next step rebuilds from scratch).
__global__ void __launch_bounds__(kPersistBlock, 8) k_rebuild(CellGrid g, SysDev s, NeighSpec ns, NeighDev cd,
                                                           DevStatus *status, GridBar *bar, int limit, int stall) {
    pdl_entry();
    if (gate_closed(s.skin)) return;
    const int G = gridDim.x;
    const int nb = (s.n + kPersistBlock - 1) / kPersistBlock;
    const int nchunk = (g.ncell + kPersistBlock - 1) / kPersistBlock;
    int *bsum = s.start + g.ncell + 1;
    auto fail = [&]() {
        if (threadIdx.x == 0) {
            atomicOr(&status->timeout, 1u);
            atomicExch(&s.skin->invalid, 1u);
        }
    };
    // counts are zero after every complete build; a build that gave up may
    // have left some, so the rebuild starts from zero
    for (int c = blockIdx.x * kPersistBlock + threadIdx.x; c < g.ncell; c += G * kPersistBlock) s.count[c] = 0;
    if (!grid_barrier(bar, limit, stall && blockIdx.x == 0)) return fail();
    for (int v = blockIdx.x; v < nb; v += G) bin_body(g, s, v);
    if (!grid_barrier(bar, limit, false)) return fail();
    for (int v = blockIdx.x; v < nchunk; v += G) scan_chunk(s, g.ncell, v, bsum);
    if (!grid_barrier(bar, limit, false)) return fail();
    for (int v = blockIdx.x; v < nchunk; v += G) scan_offset(s, g.ncell, v, nchunk, bsum);
    if (!grid_barrier(bar, limit, false)) return fail();
    for (int v = blockIdx.x; v < nb; v += G) scatter_body(s, g.ncell, v, nb);
    if (!grid_barrier(bar, limit, false)) return fail();
    for (int v = blockIdx.x; v < nb; v += G) place_body(g, s, v);
    if (!grid_barrier(bar, limit, false)) return fail();
    if (blockIdx.x == 0 && threadIdx.x == 0) s.skin->invalid = 0u;
    for (int v = blockIdx.x; v < nb; v += G) neighbors_fast_body<NK_CAND>(g, s, ns, cd, status, v);
}

}  // namespace

int rebuild_blocks() {
    static int blocks[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 0;
    if (blocks[dev] == 0) {
        int sms = 0, per = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_rebuild, kPersistBlock, 0) != cudaSuccess) return 0;
        blocks[dev] = per * sms > 0 ? per * sms : -1;
    }
    return blocks[dev] > 0 ? blocks[dev] : 0;
}

cudaError_t launch_rebuild(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev cd, DevStatus *status,
                           GridBar *bar, int limit, int stall, cudaStream_t st) {
    const int blocks = rebuild_blocks();
    if (blocks < 1) return cudaErrorInvalidConfiguration;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kPersistBlock);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_rebuild, g, s, ns, cd, status, bar, limit, stall);
    prof_mark("skin_rebuild", st);
    return e;
}

int launch_build_cells(const CellGrid &g, SysDev &s, cudaStream_t st) {
    const int nb = (s.n + kBlock - 1) / kBlock;
    const SkinState *sk = s.skin;
    if (s.n > 0) launch_k(k_bin, nb, kBlock, 0, st, g, s);
    prof_mark("cell_bin", st);
    {
        const int sb = (g.ncell + kScanBlock - 1) / kScanBlock;
        int *bsum = s.start + g.ncell + 1;   // scratch after the ncell + 1 starts
        launch_k(k_scan_blocks, sb, kScanBlock, 0, st, s.count, s.start, bsum, g.ncell, sk);
        if (sb <= kScanBlock) {
            launch_k(k_scan_add_fused, sb, kScanBlock, 0, st, s.start, bsum, g.ncell, sb, sk);
        } else {
            launch_k(k_scan_top, 1, kScanBlock, 0, st, bsum, sb, s.start, g.ncell, sk);
            launch_k(k_scan_add, sb, kScanBlock, 0, st, s.start, bsum, g.ncell, sk);
        }
    }
    prof_mark("cell_scan", st);
    if (s.n > 0) {
        launch_k(k_scatter, nb, kBlock, 0, st, s, g.ncell);
        prof_mark("cell_scatter", st);
        launch_k(k_place, nb, kBlock, 0, st, g, s);
        prof_mark("cell_sort", st);
    }
    const int sb = (g.ncell + kScanBlock - 1) / kScanBlock;
    return (s.n > 0 ? 3 : 0) + (sb <= kScanBlock ? 2 : 3);
}

void launch_neighbors(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev nd, DevStatus *status,
                      cudaStream_t st) {
    if (s.n == 0) return;
    const int nb = (s.n + kBlock - 1) / kBlock;
    bool fast = true;
    for (int c = 0; c < 3; ++c)
        if (g.periodic[c] && g.nc[c] < 3) fast = false;
    // the fast path has three interchangeable shapes (identical lists): 256- or
    // 128-thread blocks of k_neighbors_fast, or k_neighbors_flat (autotuned)
    // skin-list candidates need the fast path (the context builds them only where it applies)
    if (fast && ns.variant == 2 && s.n < (1 << 26)) {
        const int fb = (s.n + kFlatBlock - 1) / kFlatBlock;
        if (ns.kind == NK_RANGE) launch_k(k_neighbors_flat<NK_RANGE>, fb, kFlatBlock, 0, st, g, s, ns, nd, status);
        else if (ns.kind == NK_STEP) launch_k(k_neighbors_flat<NK_STEP>, fb, kFlatBlock, 0, st, g, s, ns, nd, status);
        else if (ns.kind == NK_CAND) launch_k(k_neighbors_flat<NK_CAND>, fb, kFlatBlock, 0, st, g, s, ns, nd, status);
        else launch_k(k_neighbors_flat<NK_SWITCH>, fb, kFlatBlock, 0, st, g, s, ns, nd, status);
    } else if (fast) {
        const int tb = ns.variant == 1 ? 128 : kBlock;
        const int gb = (s.n + tb - 1) / tb;
        if (ns.kind == NK_RANGE) launch_k(k_neighbors_fast<NK_RANGE>, gb, tb, 0, st, g, s, ns, nd, status);
        else if (ns.kind == NK_STEP) launch_k(k_neighbors_fast<NK_STEP>, gb, tb, 0, st, g, s, ns, nd, status);
        else if (ns.kind == NK_CAND) launch_k(k_neighbors_fast<NK_CAND>, gb, tb, 0, st, g, s, ns, nd, status);
        else launch_k(k_neighbors_fast<NK_SWITCH>, gb, tb, 0, st, g, s, ns, nd, status);
    } else if (ns.kind == NK_RANGE) launch_k(k_neighbors<NK_RANGE>, nb, kBlock, 0, st, g, s, ns, nd, status);
    else if (ns.kind == NK_STEP) launch_k(k_neighbors<NK_STEP>, nb, kBlock, 0, st, g, s, ns, nd, status);
    else launch_k(k_neighbors<NK_SWITCH>, nb, kBlock, 0, st, g, s, ns, nd, status);
    prof_mark(ns.kind == NK_CAND ? "neighbor_candidates" : "neighbors", st);
    if (ns.cap > 0 && ns.kind != NK_CAND) launch_select_cap(g, s, ns, nd, st);
}

void launch_select_cap(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev nd, cudaStream_t st) {
    if (s.n == 0) return;
    const int nb = (s.n + kBlock - 1) / kBlock;
    launch_k(k_select_cap, nb, kBlock, 0, st, g, s, ns, nd);
    prof_mark("select_cap", st);
}

void launch_refresh(const CellGrid &g, const SysDev &s, int every, double half_skin, int force, cudaStream_t st) {
    const int nb = s.n > 0 ? (s.n + kBlock - 1) / kBlock : 1;
    launch_k(k_refresh, nb, kBlock, 0, st, g, s, every, half_skin * half_skin, force);
    prof_mark("skin_refresh", st);
}

void launch_filter(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev nd, NeighDev cand,
                   DevStatus *status, SkinState *reset, cudaStream_t st) {
    const int nb = s.n > 0 ? (s.n + kBlock - 1) / kBlock : 1;
    if (ns.kind == NK_RANGE) launch_k(k_filter<NK_RANGE>, nb, kBlock, 0, st, g, s, ns, nd, cand, status, reset);
    else if (ns.kind == NK_STEP) launch_k(k_filter<NK_STEP>, nb, kBlock, 0, st, g, s, ns, nd, cand, status, reset);
    else launch_k(k_filter<NK_SWITCH>, nb, kBlock, 0, st, g, s, ns, nd, cand, status, reset);
    prof_mark("skin_filter", st);
}

}  // namespace mtd
