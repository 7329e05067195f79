// persist.cuh -- pieces of the persistent (cooperative, grid-barrier) kernels:
// the cell-count scan in 256-cell chunks and a bounded grid barrier.
//
// The persistent kernels loop over "virtual blocks" (256 atoms or 256 cells)
// with a grid-stride loop, so a phase does the same per-thread work as the
// one-block-per-item kernels it replaces, and separate phases by a grid
// barrier instead of a kernel boundary.  They are launched cooperatively (all
// blocks co-resident), so every barrier wait ends in normal operation; each
// wait still polls at most `limit` times, after which the block records the
// failure in the barrier and leaves, and every other block leaves at its
// next barrier.
#pragma once

#include "neigh_body.cuh"

namespace mtd {

constexpr int kPersistBlock = 256;

// Exclusive scan of one value per thread over a block of kPersistBlock threads.
__device__ __forceinline__ int scan256(int v, int &total) {
    __shared__ int warp_tot[kPersistBlock / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[warp] = x;
    __syncthreads();
    int before = 0;
    total = 0;
#pragma unroll
    for (int w = 0; w < kPersistBlock / 32; ++w) {
        const int t = warp_tot[w];
        if (w < warp) before += t;
        total += t;
    }
    __syncthreads();
    return before + x - v;
}

// Chunk c of the cell counts: exclusive scan into start, the chunk total into bsum[c].
__device__ __forceinline__ void scan_chunk(const SysDev &s, int ncell, int c, int *bsum) {
    const int i = c * kPersistBlock + threadIdx.x;
    int total;
    const int e = scan256(i < ncell ? s.count[i] : 0, total);
    if (i < ncell) s.start[i] = e;
    if (threadIdx.x == 0) bsum[c] = total;
}

// The totals of the chunks before c added to chunk c; the last chunk writes start[ncell].
__device__ __forceinline__ void scan_offset(const SysDev &s, int ncell, int c, int nchunk, const int *bsum) {
    __shared__ int red[kPersistBlock / 32];
    int v = 0;
    for (int t = threadIdx.x; t < c; t += kPersistBlock) v += bsum[t];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    int off = 0;
#pragma unroll
    for (int w = 0; w < kPersistBlock / 32; ++w) off += red[w];
    __syncthreads();
    const int i = c * kPersistBlock + threadIdx.x;
    if (i < ncell) s.start[i] += off;
    if (c == nchunk - 1 && threadIdx.x == 0) s.start[ncell] = off + bsum[c];
}

// Bounded grid barrier (count and generation words); false in every thread
// when this block or another gave up a wait.  stall (diagnostics): this block
// does not arrive, so the others' waits run out.
__device__ __forceinline__ bool grid_barrier(GridBar *b, int limit, bool stall) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        volatile unsigned *gen = &b->gen;
        const unsigned g = *gen;
        __threadfence();
        if (stall) {
            good = 0;
        } else if (atomicAdd(&b->count, 1u) == gridDim.x - 1) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            int it = 0;
            while (*gen == g) {
                if (++it > limit) {
                    atomicExch(&b->err, 1u);
                    good = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        __threadfence();
        ok = good && *(volatile unsigned *)&b->err == 0u;
    }
    __syncthreads();
    return ok != 0;
}

}  // namespace mtd
