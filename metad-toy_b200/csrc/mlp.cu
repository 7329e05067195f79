// mlp.cu -- learned bias V_theta(s) for CV_dim >= 3: an MLP D -> 128 -> 128 -> 1
// with SiLU activations, BF16 weights and FP32 accumulation, trained on the GPU
// on the FP64 hill sum the method deposits, which stays the measure of its error
// and the fallback.  No counterpart in the reference (its grids are the only
// bias representation: src/grids/GH_t0_uniformGrid.cu, GH_t1_sparseGrid.cu).
//
// Kernels
//   k_hillsum_batch   exact FP64 V and dV/ds for a batch of points (hill tiles in shared memory)
//   k_hillsum_point   exact FP64 V and dV/ds at one point, hills spread over the grid
//   k_mlp_tile        128 points per CTA: layer 1 and 3 on CUDA cores, the 128 x 128
//                     layer and its two backward contractions on tcgen05 (TMEM accumulators)
//   k_mlp_adam        sums the per-tile gradients in tile order, Adam step, BF16 copies
//   k_mlp_point       V_theta and dV_theta/ds at one point (CUDA cores, one block)
//
// Network on normalised inputs u = 2 (s - lo) / (hi - lo) - 1 and outputs
// V = vscale * y:  z1 = W1 u + b1, h1 = silu(z1), z2 = W2 h1 + b2,
// h2 = silu(z2), y = w3 . h2 + b3.  W1, W2, w3 are used as BF16 values
// (FP32 masters for Adam); h1 and dL/dz2 are rounded to BF16 as tensor-core
// operands, every sum accumulates in FP32.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/metad_b200.h"
#include "common.cuh"
#include "umma.cuh"

namespace mtd {

namespace {

constexpr int kH = 128;                 // hidden width
constexpr int kIn = 4;                  // input slots (D <= 4)
constexpr int oW1 = 0;                  // flat parameter layout
constexpr int ob1 = oW1 + kH * kIn;
constexpr int oW2 = ob1 + kH;
constexpr int ob2 = oW2 + kH * kH;
constexpr int ow3 = ob2 + kH;
constexpr int ob3 = ow3 + kH;
constexpr int kNP = ob3 + 1;            // 17,281 parameters
constexpr int kNPpad = (kNP + 3) / 4 * 4;
constexpr int kTileSmem = 6 * 32768 + (4 * kH + 3 * kH) * 4 + 64;   // operand tiles + small weights
constexpr int kWaitTries = 1 << 20;     // bounded mbarrier waits (default limit)

enum { MODE_FWD = 0, MODE_GRAD_S = 1, MODE_TRAIN = 2 };

struct MlpDev {
    int D;
    const float *W1, *b1, *b2, *w3, *b3;       // W1, w3: BF16-rounded values
    const __nv_bfloat16 *W2, *W2t;             // [n][k] and [k][n]
};

__device__ __forceinline__ float silu(float z, float &dsilu) {
    const float s = 1.0f / (1.0f + __expf(-z));
    dsilu = s * (1.0f + z * (1.0f - s));
    return z * s;
}

// Sum over the 128 rows of a CTA of Q per-row values, Q <= 96: rows write a
// [128][Q+1] FP32 tile, then thread q sums column q in row order.
__device__ __forceinline__ void rows_sum(float *scratch, const float *vals, int Q, float *out) {
    const int m = threadIdx.x;
    for (int q = 0; q < Q; ++q) scratch[m * (Q + 1) + q] = vals[q];
    __syncthreads();
    if (m < Q) {
        float s = 0.0f;
        for (int r = 0; r < kH; ++r) s += scratch[r * (Q + 1) + m];
        out[m] = s;
    }
    __syncthreads();
}

// A bounded wait that runs out (in any thread: the block votes) ends the
// tile: it issues no further MMA, reads no TMEM and overlays no operand the
// tensor core may still be reading; it waits once more (same limit) for the
// batch in flight, releases its TMEM, sets *err and returns.  stall != 0 is
// the check of that path: after the first batch has completed, every thread
// waits on the barrier's next phase, which no commit will complete.
template <int MODE>
__global__ void __launch_bounds__(128, 1)
    k_mlp_tile(MlpDev p, int npts, const float *__restrict__ x, const float *__restrict__ t, float *y_out,
               float *ds_out, float *part, float *loss_part, float grad_scale, int *err, int tries, int stall) {
    extern __shared__ __align__(1024) unsigned char sm[];
    unsigned char *sA = sm;                   // h1        rows m, K k
    unsigned char *sBf = sm + 32768;          // W2        rows n, K k
    unsigned char *sBt = sm + 2 * 32768;      // W2^T      rows k, K n
    unsigned char *sG = sm + 3 * 32768;       // dL/dz2    rows m, K n
    unsigned char *sGt = sm + 4 * 32768;      // dL/dz2^T  rows n, K m
    unsigned char *sHt = sm + 5 * 32768;      // h1^T      rows k, K m
    float *sW1 = reinterpret_cast<float *>(sm + 6 * 32768);
    float *sb1 = sW1 + 4 * kH, *sb2 = sb1 + kH, *sw3 = sb2 + kH;
    float *scratch = reinterpret_cast<float *>(sm);   // reused once the operands are consumed
    __shared__ uint64_t mbar;
    __shared__ uint32_t tbase;
    __shared__ float cols[96];
    const int m = threadIdx.x, warp = m >> 5;
    const int row = blockIdx.x * kH + m;
    const bool valid = row < npts;

    if (m == 0) mbar_init(&mbar, 1);
    if (warp == 0) tmem_alloc(&tbase, 512);
    tc_fence_before();
    // weights: W2 and W2^T rows as 16-byte vectors into the operand layout
    {
        const uint4 *w2 = reinterpret_cast<const uint4 *>(p.W2 + (size_t)m * kH);
        const uint4 *w2t = reinterpret_cast<const uint4 *>(p.W2t + (size_t)m * kH);
#pragma unroll 4
        for (int c = 0; c < kH / 8; ++c) {
            *reinterpret_cast<uint4 *>(sBf + umma_off(m, 8 * c, kH)) = w2[c];
            *reinterpret_cast<uint4 *>(sBt + umma_off(m, 8 * c, kH)) = w2t[c];
        }
        for (int i = 0; i < kIn; ++i) sW1[m * kIn + i] = p.W1[m * kIn + i];
        sb1[m] = p.b1[m];
        sb2[m] = p.b2[m];
        sw3[m] = p.w3[m];
    }
    __syncthreads();
    float u[kIn] = {0.f, 0.f, 0.f, 0.f};
    if (valid)
        for (int i = 0; i < p.D; ++i) u[i] = x[(size_t)row * kIn + i];
    // layer 1 -> h1 (BF16) in the A layout, and h1^T for the weight gradient
    for (int c = 0; c < kH / 8; ++c) {
        __align__(16) __nv_bfloat16 hb[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
            const int j = 8 * c + e;
            float z = sb1[j];
#pragma unroll
            for (int i = 0; i < kIn; ++i) z = fmaf(sW1[j * kIn + i], u[i], z);
            float ds;
            hb[e] = __float2bfloat16_rn(silu(z, ds));
            if (MODE == MODE_TRAIN) *reinterpret_cast<__nv_bfloat16 *>(sHt + umma_off(j, m, kH)) = hb[e];
        }
        *reinterpret_cast<uint4 *>(sA + umma_off(m, 8 * c, kH)) = *reinterpret_cast<const uint4 *>(hb);
    }
    fence_async_smem();
    __syncthreads();
    tc_fence_after();
    const uint32_t taddr = tbase;
    const uint32_t idesc = umma_idesc_bf16(kH, kH);
    if (m == 0) {
        for (int kk = 0; kk < kH / 16; ++kk) {
            const uint64_t a = umma_desc(smem_addr(sA) + kk * 2 * kH * 16, kH * 16, 128);
            const uint64_t b = umma_desc(smem_addr(sBf) + kk * 2 * kH * 16, kH * 16, 128);
            umma_bf16(taddr, a, b, idesc, kk > 0 ? 1u : 0u);
        }
        umma_commit(&mbar);
    }
    bool ok = mbar_wait(&mbar, 0, tries);
    if (stall) ok = mbar_wait(&mbar, 1, tries) && ok;
    if (!__syncthreads_and(ok)) {
        mbar_wait(&mbar, 0, tries);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(taddr, 512);
        if (m == 0) atomicExch(err, 1);
        return;
    }
    tc_fence_after();
    const uint32_t lane_addr = taddr + (static_cast<uint32_t>(warp * 32) << 16);
    // forward epilogue: z2 = D + b2, y = w3 . silu(z2) + b3
    float y = p.b3[0];
    for (int c = 0; c < kH / 16; ++c) {
        float z[16];
        tmem_ld16(lane_addr + 16 * c, z);
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            float ds;
            y = fmaf(sw3[16 * c + e], silu(z[e] + sb2[16 * c + e], ds), y);
        }
    }
    if (valid && y_out) y_out[row] = y;
    if (MODE == MODE_FWD) {
        tc_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(taddr, 512);
        return;
    }
    float dy = 0.0f;
    if (valid) dy = (MODE == MODE_TRAIN) ? grad_scale * (y - t[row]) : 1.0f;
    if (MODE == MODE_TRAIN) {
        float l = valid ? (y - t[row]) * (y - t[row]) : 0.0f;
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if ((m & 31) == 0) cols[warp] = l;
        __syncthreads();
        if (m == 0) loss_part[blockIdx.x] = cols[0] + cols[1] + cols[2] + cols[3];
        __syncthreads();
    }
    // dL/dz2 = dy w3 silu'(z2): BF16 into the A layout (and its transpose);
    // b2, w3 gradients summed over rows in FP32
    for (int c = 0; c < kH / 16; ++c) {
        float z[16];
        tmem_ld16(lane_addr + 16 * c, z);
        __align__(16) __nv_bfloat16 gb[16];
        float red[32];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int n = 16 * c + e;
            float dsl;
            const float h2 = silu(z[e] + sb2[n], dsl);
            const float g = dy * sw3[n] * dsl;
            gb[e] = __float2bfloat16_rn(g);
            red[e] = g;
            red[16 + e] = dy * h2;
            if (MODE == MODE_TRAIN) *reinterpret_cast<__nv_bfloat16 *>(sGt + umma_off(n, m, kH)) = gb[e];
        }
        *reinterpret_cast<uint4 *>(sG + umma_off(m, 16 * c, kH)) = *reinterpret_cast<const uint4 *>(gb);
        *reinterpret_cast<uint4 *>(sG + umma_off(m, 16 * c + 8, kH)) = *reinterpret_cast<const uint4 *>(gb + 8);
        if (MODE == MODE_TRAIN) {
            // scratch overlays sA / sBf, free since the forward MMA completed
            rows_sum(scratch, red, 32, cols);
            if (m < 16) part[(size_t)blockIdx.x * kNPpad + ob2 + 16 * c + m] = cols[m];
            else if (m < 32) part[(size_t)blockIdx.x * kNPpad + ow3 + 16 * c + (m - 16)] = cols[m];
        }
    }
    if (MODE == MODE_TRAIN) {
        float v[1] = {dy};
        rows_sum(scratch, v, 1, cols);
        if (m == 0) part[(size_t)blockIdx.x * kNPpad + ob3] = cols[0];
    }
    fence_async_smem();
    __syncthreads();
    tc_fence_after();
    if (m == 0) {
        for (int kk = 0; kk < kH / 16; ++kk) {   // dL/dh1 = dL/dz2 . W2  -> columns 128..255
            const uint64_t a = umma_desc(smem_addr(sG) + kk * 2 * kH * 16, kH * 16, 128);
            const uint64_t b = umma_desc(smem_addr(sBt) + kk * 2 * kH * 16, kH * 16, 128);
            umma_bf16(taddr + kH, a, b, idesc, kk > 0 ? 1u : 0u);
        }
        if (MODE == MODE_TRAIN) {
            for (int kk = 0; kk < kH / 16; ++kk) {   // dL/dW2 = dL/dz2^T . h1  -> columns 256..383
                const uint64_t a = umma_desc(smem_addr(sGt) + kk * 2 * kH * 16, kH * 16, 128);
                const uint64_t b = umma_desc(smem_addr(sHt) + kk * 2 * kH * 16, kH * 16, 128);
                umma_bf16(taddr + 2 * kH, a, b, idesc, kk > 0 ? 1u : 0u);
            }
        }
        umma_commit(&mbar);
    }
    if (!__syncthreads_and(mbar_wait(&mbar, 1, tries))) {
        mbar_wait(&mbar, 1, tries);
        tc_fence_before();
        __syncthreads();
        if (warp == 0) tmem_dealloc(taddr, 512);
        if (m == 0) atomicExch(err, 1);
        return;
    }
    tc_fence_after();
    // layer 1 backward: dL/dz1 = dL/dh1 silu'(z1); input gradient and W1, b1 gradients
    float dsu[kIn] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < kH / 16; ++c) {
        float dh[16];
        tmem_ld16(lane_addr + kH + 16 * c, dh);
        float red[80];
#pragma unroll
        for (int e = 0; e < 16; ++e) {
            const int j = 16 * c + e;
            float z = sb1[j];
#pragma unroll
            for (int i = 0; i < kIn; ++i) z = fmaf(sW1[j * kIn + i], u[i], z);
            float dsl;
            silu(z, dsl);
            const float g = dh[e] * dsl;
#pragma unroll
            for (int i = 0; i < kIn; ++i) {
                dsu[i] = fmaf(g, sW1[j * kIn + i], dsu[i]);
                red[16 + 16 * i + e] = g * u[i];
            }
            red[e] = g;
        }
        if (MODE == MODE_TRAIN) {
            rows_sum(scratch, red, 80, cols);
            if (m < 16) part[(size_t)blockIdx.x * kNPpad + ob1 + 16 * c + m] = cols[m];
            else if (m < 80) {
                const int i = (m - 16) >> 4, e = (m - 16) & 15;
                part[(size_t)blockIdx.x * kNPpad + oW1 + (16 * c + e) * kIn + i] = cols[m];
            }
        }
    }
    if (MODE == MODE_GRAD_S && valid && ds_out)
        for (int i = 0; i < kIn; ++i) ds_out[(size_t)row * kIn + i] = dsu[i];
    if (MODE == MODE_TRAIN) {   // row n of the W2 gradient
        float *dst = part + (size_t)blockIdx.x * kNPpad + oW2 + (size_t)m * kH;
        for (int c = 0; c < kH / 16; ++c) {
            float g[16];
            tmem_ld16(lane_addr + 2 * kH + 16 * c, g);
#pragma unroll
            for (int e = 0; e < 16; ++e) dst[16 * c + e] = g[e];
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_dealloc(taddr, 512);
}

__device__ __forceinline__ float bf16_round(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// Adam on the FP32 masters with the gradient summed over tiles in tile order;
// refreshes the forward copies (BF16 W1, W2, W2^T, w3; FP32 biases).
__global__ void k_mlp_adam(int ntiles, const float *__restrict__ part, float *master, float *mom, float *vel,
                           float lr, float b1c, float b2c, float *W1, float *b1, __nv_bfloat16 *W2,
                           __nv_bfloat16 *W2t, float *b2, float *w3, float *b3, int update) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kNP) return;
    float w = master[q];
    if (update) {
        float g = 0.0f;
        for (int t = 0; t < ntiles; ++t) g += part[(size_t)t * kNPpad + q];
        const float m1 = 0.9f * mom[q] + 0.1f * g;
        const float v1 = 0.999f * vel[q] + 0.001f * g * g;
        mom[q] = m1;
        vel[q] = v1;
        w -= lr * (m1 / b1c) / (sqrtf(v1 / b2c) + 1e-8f);
        master[q] = w;
    }
    if (q < ob1) W1[q] = bf16_round(w);
    else if (q < oW2) b1[q - ob1] = w;
    else if (q < ob2) {
        const int n = (q - oW2) / kH, k = (q - oW2) % kH;
        W2[n * kH + k] = __float2bfloat16_rn(w);
        W2t[k * kH + n] = __float2bfloat16_rn(w);
    } else if (q < ow3) b2[q - ob2] = w;
    else if (q < ob3) w3[q - ow3] = bf16_round(w);
    else b3[0] = w;
}

// Gradient summed over tiles without an update (for checks).
__global__ void k_mlp_gradsum(int ntiles, const float *__restrict__ part, float *g) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kNP) return;
    float s = 0.0f;
    for (int t = 0; t < ntiles; ++t) s += part[(size_t)t * kNPpad + q];
    g[q] = s;
}

// Hills packed as [c0 c1 c2 c3 w 1/(2 sigma^2) 1/sigma^2 0] (FP64).  A hill
// farther than sqrt(80) sigma from the point contributes below h e^-40
// (4e-18 h) and is skipped; its gradient term is smaller still.
constexpr int kHillTile = 256;
constexpr double kExpCut = 40.0;

// Points and gradients are rows of `ps` / `gs` doubles (kIn, or D for caller
// layouts); a gradient row of D < gs leaves the rest unwritten.
__global__ void __launch_bounds__(256) k_hillsum_batch(int D, int npts, const double *__restrict__ pts, int ps, int nh,
                                                       const double *__restrict__ hills, double *V, double *dV,
                                                       int gs) {
    __shared__ double sh[kHillTile * 8];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s[kIn] = {0, 0, 0, 0};
    if (i < npts)
        for (int k = 0; k < D; ++k) s[k] = pts[(size_t)i * ps + k];
    double v = 0.0, g[kIn] = {0, 0, 0, 0};
    for (int h0 = 0; h0 < nh; h0 += kHillTile) {
        const int nt = min(kHillTile, nh - h0);
        __syncthreads();
        for (int e = threadIdx.x; e < nt * 8; e += blockDim.x) sh[e] = hills[(size_t)h0 * 8 + e];
        __syncthreads();
        for (int h = 0; h < nt; ++h) {
            const double *c = sh + 8 * h;
            double r2 = 0.0, d[kIn];
#pragma unroll
            for (int k = 0; k < kIn; ++k) {
                d[k] = k < D ? s[k] - c[k] : 0.0;
                r2 += d[k] * d[k];
            }
            const double a = r2 * c[5];
            if (a < kExpCut) {
                const double e = c[4] * exp(-a);
                v += e;
#pragma unroll
                for (int k = 0; k < kIn; ++k) g[k] -= e * d[k] * c[6];
            }
        }
    }
    if (i < npts) {
        V[i] = v;
        if (dV)
            for (int k = 0; k < min(gs, kIn); ++k)
                if (k < D || gs == kIn) dV[(size_t)i * gs + k] = g[k];
    }
}

// Caller points (rows of D doubles) to the network's normalised FP32 inputs.
__global__ void k_nb_inputs(int D, int npts, const double *__restrict__ pts, double lo0, double lo1, double lo2,
                            double lo3, double sc0, double sc1, double sc2, double sc3, float *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npts) return;
    const double lo[kIn] = {lo0, lo1, lo2, lo3}, sc[kIn] = {sc0, sc1, sc2, sc3};
#pragma unroll
    for (int k = 0; k < kIn; ++k) x[(size_t)i * kIn + k] = k < D ? (float)(sc[k] * (pts[(size_t)i * D + k] - lo[k]) - 1.0) : 0.f;
}

// Network outputs to V = vscale y and dV/ds = vscale dy/du du/ds (FP64, rows of D).
__global__ void k_nb_outputs(int D, int npts, const float *__restrict__ y, const float *__restrict__ ds,
                             double vscale, double sc0, double sc1, double sc2, double sc3, double *V, double *dV) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npts) return;
    const double sc[kIn] = {sc0, sc1, sc2, sc3};
    V[i] = vscale * (double)y[i];
    if (dV)
        for (int k = 0; k < D; ++k) dV[(size_t)i * D + k] = vscale * (double)ds[(size_t)i * kIn + k] * sc[k];
}

// One point, hills spread over blocks; block partials reduced in block order by the last block.
constexpr int kPointBlocks = 80;
__global__ void __launch_bounds__(256) k_hillsum_point(int D, const double *__restrict__ s_in, int h_begin, int nh,
                                                       const double *__restrict__ hills, double *part,
                                                       unsigned int *ticket, double *V, double *dV,
                                                       int accumulate) {
    __shared__ double smem[5 * 32];
    __shared__ bool last;
    double s[kIn] = {0, 0, 0, 0};
    for (int k = 0; k < D; ++k) s[k] = s_in[k];
    double acc[5] = {0, 0, 0, 0, 0};
    for (int h = h_begin + blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += gridDim.x * blockDim.x) {
        const double *c = hills + (size_t)h * 8;
        double r2 = 0.0, d[kIn];
#pragma unroll
        for (int k = 0; k < kIn; ++k) {
            d[k] = k < D ? s[k] - c[k] : 0.0;
            r2 += d[k] * d[k];
        }
        const double a = r2 * c[5];
        if (a < kExpCut) {
            const double e = c[4] * exp(-a);
            acc[0] += e;
#pragma unroll
            for (int k = 0; k < kIn; ++k) acc[1 + k] -= e * d[k] * c[6];
        }
    }
    block_sum<5>(acc, smem);
    if (threadIdx.x == 0) {
        for (int q = 0; q < 5; ++q) part[blockIdx.x * 5 + q] = acc[q];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x < 5) {
        __threadfence();
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) t += *((volatile double *)part + b * 5 + threadIdx.x);
        if (threadIdx.x == 0) *V = accumulate ? *V + t : t;
        else if ((int)threadIdx.x - 1 < D) dV[threadIdx.x - 1] = accumulate ? dV[threadIdx.x - 1] + t : t;
        if (threadIdx.x == 0) *ticket = 0u;
    }
}

// V_theta and dV_theta/ds at one point (FP64 in/out), one block of 128 threads.
__global__ void __launch_bounds__(128) k_mlp_point(MlpDev p, const double *__restrict__ s_in, double lo0, double lo1,
                                                   double lo2, double lo3, double sc0, double sc1, double sc2,
                                                   double sc3, double vscale, double *V, double *dV) {
    __shared__ float h1[kH], dz2[kH], red[kIn + 1][4];
    const int j = threadIdx.x, warp = j >> 5;
    const double lo[kIn] = {lo0, lo1, lo2, lo3}, sc[kIn] = {sc0, sc1, sc2, sc3};   // sc = 2 / (hi - lo)
    float u[kIn] = {0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < p.D; ++i) u[i] = (float)((s_in[i] - lo[i]) * sc[i] - 1.0);
    float z1 = p.b1[j];
    for (int i = 0; i < kIn; ++i) z1 = fmaf(p.W1[j * kIn + i], u[i], z1);
    float ds1;
    h1[j] = __bfloat162float(__float2bfloat16_rn(silu(z1, ds1)));
    __syncthreads();
    float z2 = p.b2[j];
    const uint4 *w = reinterpret_cast<const uint4 *>(p.W2 + (size_t)j * kH);   // row j, 8 BF16 per load
    uint4 wv[kH / 8];
#pragma unroll
    for (int c = 0; c < kH / 8; ++c) wv[c] = __ldg(w + c);
#pragma unroll
    for (int c = 0; c < kH / 8; ++c) {
        const __nv_bfloat162 *pr = reinterpret_cast<const __nv_bfloat162 *>(&wv[c]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 f = __bfloat1622float2(pr[e]);
            z2 = fmaf(f.x, h1[8 * c + 2 * e], z2);
            z2 = fmaf(f.y, h1[8 * c + 2 * e + 1], z2);
        }
    }
    float ds2;
    const float h2 = silu(z2, ds2);
    float yv = p.w3[j] * h2;
    dz2[j] = __bfloat162float(__float2bfloat16_rn(p.w3[j] * ds2));
    __syncthreads();
    float dh = 0.0f;
    const uint4 *wt = reinterpret_cast<const uint4 *>(p.W2t + (size_t)j * kH);
#pragma unroll
    for (int c = 0; c < kH / 8; ++c) wv[c] = __ldg(wt + c);
#pragma unroll
    for (int c = 0; c < kH / 8; ++c) {
        const __nv_bfloat162 *pr = reinterpret_cast<const __nv_bfloat162 *>(&wv[c]);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const float2 f = __bfloat1622float2(pr[e]);
            dh = fmaf(f.x, dz2[8 * c + 2 * e], dh);
            dh = fmaf(f.y, dz2[8 * c + 2 * e + 1], dh);
        }
    }
    const float g = dh * ds1;
    float q[kIn + 1] = {yv, 0.f, 0.f, 0.f, 0.f};
    for (int i = 0; i < kIn; ++i) q[1 + i] = g * p.W1[j * kIn + i];
    for (int t = 0; t < kIn + 1; ++t)
        for (int o = 16; o > 0; o >>= 1) q[t] += __shfl_xor_sync(0xffffffffu, q[t], o);
    if ((j & 31) == 0)
        for (int t = 0; t < kIn + 1; ++t) red[t][warp] = q[t];
    __syncthreads();
    if (j < kIn + 1) {
        const float s = red[j][0] + red[j][1] + red[j][2] + red[j][3];
        if (j == 0) *V = vscale * (double)(s + p.b3[0]);
        else if (j - 1 < p.D) dV[j - 1] = vscale * (double)s * sc[j - 1];
    }
}

}  // namespace

}  // namespace mtd

// ------------------------------------------------------------------ host object
using namespace mtd;

struct mtd_nnbias {
    int D = 0, device = 0;
    double lo[kIn] = {0, 0, 0, 0}, hi[kIn] = {1, 1, 1, 1};
    double vscale = 1.0;
    cudaStream_t st = nullptr;
    std::string err;
    std::vector<double> hills;   // packed, 8 doubles per hill
    double *d_hills = nullptr;
    int nh = 0, cap_h = 0;
    float *d_master = nullptr, *d_mom = nullptr, *d_vel = nullptr;
    float *d_W1 = nullptr, *d_b1 = nullptr, *d_b2 = nullptr, *d_w3 = nullptr, *d_b3 = nullptr;
    __nv_bfloat16 *d_W2 = nullptr, *d_W2t = nullptr;
    float *d_part = nullptr, *d_loss = nullptr;
    int cap_tiles = 0;
    int adam_t = 0;
    int *d_err = nullptr;
    double *d_pt = nullptr, *d_ppart = nullptr, *d_pout = nullptr;
    // device batch evaluation scratch (grown on demand)
    float *d_bx = nullptr, *d_by = nullptr, *d_bds = nullptr;
    int cap_b = 0;
    unsigned int *d_ticket = nullptr;
    // training pool
    int ntrain = 0;
    float *d_xt = nullptr, *d_tt = nullptr;
    bool validated = false;
    double tol = 1e-3, last_max_err = -1.0;
    unsigned long long seed = 1;
    int wait_tries = kWaitTries;   // limit of the tile kernel's mbarrier waits
    int wait_stall = 0;            // 1: tiles take their timeout path (mtd_nnbias_set_wait)
};

namespace {

std::mutex g_attr_mutex;
bool g_attr_done[64] = {};

mtd_status nb_fail(mtd_nnbias *b, mtd_status s, const std::string &m) {
    if (b) b->err = m;
    return s;
}

#define NB_CU(call, what)                                                                          \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            return nb_fail(b, e_ == cudaErrorMemoryAllocation ? MTD_ERR_OOM : MTD_ERR_CUDA,        \
                           std::string(what) + ": " + cudaGetErrorString(e_));                     \
    } while (0)

MlpDev nb_dev(const mtd_nnbias *b) {
    MlpDev p;
    p.D = b->D;
    p.W1 = b->d_W1;
    p.b1 = b->d_b1;
    p.b2 = b->d_b2;
    p.w3 = b->d_w3;
    p.b3 = b->d_b3;
    p.W2 = b->d_W2;
    p.W2t = b->d_W2t;
    return p;
}

mtd_status nb_tile_attr(mtd_nnbias *b) {
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    if (b->device >= 0 && b->device < 64 && g_attr_done[b->device]) return MTD_OK;
    NB_CU(cudaFuncSetAttribute(k_mlp_tile<MODE_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem),
          "smem attribute");
    NB_CU(cudaFuncSetAttribute(k_mlp_tile<MODE_GRAD_S>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem),
          "smem attribute");
    NB_CU(cudaFuncSetAttribute(k_mlp_tile<MODE_TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem),
          "smem attribute");
    if (b->device >= 0 && b->device < 64) g_attr_done[b->device] = true;
    return MTD_OK;
}

mtd_status nb_ensure_tiles(mtd_nnbias *b, int ntiles) {
    if (ntiles <= b->cap_tiles) return MTD_OK;
    if (b->d_part) cudaFree(b->d_part);
    if (b->d_loss) cudaFree(b->d_loss);
    b->d_part = nullptr;
    b->d_loss = nullptr;
    NB_CU(cudaMalloc(&b->d_part, sizeof(float) * (size_t)kNPpad * ntiles), "gradient partials");
    NB_CU(cudaMalloc(&b->d_loss, sizeof(float) * (size_t)ntiles), "loss partials");
    b->cap_tiles = ntiles;
    return MTD_OK;
}

void nb_normalise(const mtd_nnbias *b, const double *s, float *u) {
    for (int i = 0; i < kIn; ++i)
        u[i] = i < b->D ? (float)(2.0 * (s[i] - b->lo[i]) / (b->hi[i] - b->lo[i]) - 1.0) : 0.0f;
}

mtd_status nb_refresh_forward(mtd_nnbias *b) {
    k_mlp_adam<<<(kNP + 255) / 256, 256, 0, b->st>>>(0, b->d_part, b->d_master, b->d_mom, b->d_vel, 0.f, 1.f, 1.f,
                                                     b->d_W1, b->d_b1, b->d_W2, b->d_W2t, b->d_b2, b->d_w3,
                                                     b->d_b3, 0);
    NB_CU(cudaGetLastError(), "forward copies");
    return MTD_OK;
}

// Exact FP64 V (and dV) at host points, computed on the device.
mtd_status nb_exact_host(mtd_nnbias *b, int npts, const double *pts, double *V, double *dV) {
    if (npts <= 0) return MTD_OK;
    std::vector<double> p4((size_t)npts * kIn, 0.0);
    for (int i = 0; i < npts; ++i)
        for (int k = 0; k < b->D; ++k) p4[(size_t)i * kIn + k] = pts[(size_t)i * b->D + k];
    double *d_p = nullptr, *d_V = nullptr, *d_dV = nullptr;
    NB_CU(cudaMalloc(&d_p, sizeof(double) * p4.size()), "points");
    NB_CU(cudaMalloc(&d_V, sizeof(double) * npts), "values");
    NB_CU(cudaMalloc(&d_dV, sizeof(double) * (size_t)npts * kIn), "gradients");
    cudaMemcpyAsync(d_p, p4.data(), sizeof(double) * p4.size(), cudaMemcpyHostToDevice, b->st);
    k_hillsum_batch<<<(npts + 255) / 256, 256, 0, b->st>>>(b->D, npts, d_p, kIn, b->nh, b->d_hills, d_V, d_dV,
                                                           kIn);
    std::vector<double> g((size_t)npts * kIn);
    cudaMemcpyAsync(V, d_V, sizeof(double) * npts, cudaMemcpyDeviceToHost, b->st);
    cudaMemcpyAsync(g.data(), d_dV, sizeof(double) * g.size(), cudaMemcpyDeviceToHost, b->st);
    const cudaError_t e = cudaStreamSynchronize(b->st);
    cudaFree(d_p);
    cudaFree(d_V);
    cudaFree(d_dV);
    NB_CU(e, "exact hill sum");
    if (dV)
        for (int i = 0; i < npts; ++i)
            for (int k = 0; k < b->D; ++k) dV[(size_t)i * b->D + k] = g[(size_t)i * kIn + k];
    return MTD_OK;
}

// Points for training / validation: half near hill centres (N(0, 1.5 sigma)),
// half uniform in the CV box.
void nb_sample(const mtd_nnbias *b, int npts, unsigned long long seed, std::vector<double> &out) {
    std::mt19937_64 g(seed);
    std::uniform_real_distribution<double> U(0.0, 1.0);
    std::normal_distribution<double> N(0.0, 1.0);
    out.assign((size_t)npts * b->D, 0.0);
    for (int i = 0; i < npts; ++i) {
        const bool near = b->nh > 0 && (i & 1);
        const int h = near ? (int)(U(g) * b->nh) % b->nh : 0;
        for (int k = 0; k < b->D; ++k) {
            double v;
            if (near) {
                const double sig = std::sqrt(1.0 / b->hills[(size_t)h * 8 + 6]);
                v = b->hills[(size_t)h * 8 + k] + 1.5 * sig * N(g);
            } else {
                v = b->lo[k] + (b->hi[k] - b->lo[k]) * U(g);
            }
            out[(size_t)i * b->D + k] = std::min(b->hi[k], std::max(b->lo[k], v));
        }
    }
}

mtd_status nb_forward_batch(mtd_nnbias *b, int npts, const float *d_x, float *d_y, float *d_ds) {
    mtd_status s = nb_tile_attr(b);
    if (s != MTD_OK) return s;
    const int ntiles = (npts + kH - 1) / kH;
    if (d_ds)
        k_mlp_tile<MODE_GRAD_S><<<ntiles, 128, kTileSmem, b->st>>>(nb_dev(b), npts, d_x, nullptr, d_y, d_ds,
                                                                   nullptr, nullptr, 0.f, b->d_err, b->wait_tries,
                                                                   b->wait_stall);
    else
        k_mlp_tile<MODE_FWD><<<ntiles, 128, kTileSmem, b->st>>>(nb_dev(b), npts, d_x, nullptr, d_y, nullptr, nullptr,
                                                                nullptr, 0.f, b->d_err, b->wait_tries,
                                                                b->wait_stall);
    NB_CU(cudaGetLastError(), "MLP forward");
    return MTD_OK;
}

// Reads and clears the tile kernels' timeout flag.
mtd_status nb_check_err(mtd_nnbias *b) {
    int h = 0;
    NB_CU(cudaMemcpyAsync(&h, b->d_err, sizeof(int), cudaMemcpyDeviceToHost, b->st), "status");
    NB_CU(cudaStreamSynchronize(b->st), "sync");
    if (h) {
        NB_CU(cudaMemsetAsync(b->d_err, 0, sizeof(int), b->st), "status");
        return nb_fail(b, MTD_ERR_TIMEOUT, "tensor-core wait ran out of tries");
    }
    return MTD_OK;
}

}  // namespace

extern "C" {

mtd_status mtd_nnbias_create(int D, const double *lo, const double *hi, unsigned long long seed, mtd_nnbias **out) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    mtd_nnbias *b = new mtd_nnbias();
    *out = b;
    if (D < 1 || D > kIn || !lo || !hi) return nb_fail(b, MTD_ERR_INVALID_ARG, "D must be in [1, 4] with lo, hi");
    b->D = D;
    for (int k = 0; k < D; ++k) {
        if (!(hi[k] > lo[k])) return nb_fail(b, MTD_ERR_INVALID_ARG, "hi must exceed lo in every dimension");
        b->lo[k] = lo[k];
        b->hi[k] = hi[k];
    }
    b->seed = seed;
    NB_CU(cudaGetDevice(&b->device), "device");
    NB_CU(cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking), "stream");
    NB_CU(cudaMalloc(&b->d_master, sizeof(float) * kNPpad), "params");
    NB_CU(cudaMalloc(&b->d_mom, sizeof(float) * kNPpad), "params");
    NB_CU(cudaMalloc(&b->d_vel, sizeof(float) * kNPpad), "params");
    NB_CU(cudaMalloc(&b->d_W1, sizeof(float) * kH * kIn), "params");
    NB_CU(cudaMalloc(&b->d_b1, sizeof(float) * kH), "params");
    NB_CU(cudaMalloc(&b->d_b2, sizeof(float) * kH), "params");
    NB_CU(cudaMalloc(&b->d_w3, sizeof(float) * kH), "params");
    NB_CU(cudaMalloc(&b->d_b3, sizeof(float) * 4), "params");
    NB_CU(cudaMalloc(&b->d_W2, sizeof(__nv_bfloat16) * kH * kH), "params");
    NB_CU(cudaMalloc(&b->d_W2t, sizeof(__nv_bfloat16) * kH * kH), "params");
    NB_CU(cudaMalloc(&b->d_err, sizeof(int)), "status");
    NB_CU(cudaMalloc(&b->d_pt, sizeof(double) * 8), "point");
    NB_CU(cudaMalloc(&b->d_pout, sizeof(double) * 8), "point");
    NB_CU(cudaMalloc(&b->d_ppart, sizeof(double) * 5 * kPointBlocks), "point partials");
    NB_CU(cudaMalloc(&b->d_ticket, sizeof(unsigned int)), "ticket");
    cudaMemsetAsync(b->d_err, 0, sizeof(int), b->st);
    cudaMemsetAsync(b->d_ticket, 0, sizeof(unsigned int), b->st);
    // He-style initialisation of the masters, zero biases
    std::vector<float> w(kNPpad, 0.0f);
    std::mt19937_64 g(seed);
    std::normal_distribution<double> N(0.0, 1.0);
    for (int j = 0; j < kH; ++j)
        for (int i = 0; i < kIn; ++i) w[oW1 + j * kIn + i] = i < D ? (float)(N(g) * std::sqrt(2.0 / D)) : 0.0f;
    for (int q = 0; q < kH * kH; ++q) w[oW2 + q] = (float)(N(g) * std::sqrt(2.0 / kH));
    for (int q = 0; q < kH; ++q) w[ow3 + q] = (float)(N(g) * std::sqrt(1.0 / kH));
    NB_CU(cudaMemcpyAsync(b->d_master, w.data(), sizeof(float) * kNPpad, cudaMemcpyHostToDevice, b->st), "init");
    cudaMemsetAsync(b->d_mom, 0, sizeof(float) * kNPpad, b->st);
    cudaMemsetAsync(b->d_vel, 0, sizeof(float) * kNPpad, b->st);
    mtd_status s = nb_refresh_forward(b);
    if (s != MTD_OK) return s;
    NB_CU(cudaStreamSynchronize(b->st), "init");
    return MTD_OK;
}

void mtd_nnbias_destroy(mtd_nnbias *b) {
    if (!b) return;
    if (b->st) cudaStreamSynchronize(b->st);
    void *ptrs[] = {b->d_hills, b->d_master, b->d_mom, b->d_vel, b->d_W1, b->d_b1, b->d_b2, b->d_w3, b->d_b3,
                    b->d_W2, b->d_W2t, b->d_part, b->d_loss, b->d_err, b->d_pt, b->d_pout, b->d_ppart,
                    b->d_ticket, b->d_xt, b->d_tt, b->d_bx, b->d_by, b->d_bds};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (b->st) cudaStreamDestroy(b->st);
    delete b;
}

const char *mtd_nnbias_last_error(const mtd_nnbias *b) { return b ? b->err.c_str() : "null object"; }

mtd_status mtd_nnbias_add_hills(mtd_nnbias *b, int n, const double *centers, const double *heights,
                                const double *sigmas) {
    if (!b || n < 0 || (n > 0 && (!centers || !heights || !sigmas))) return MTD_ERR_INVALID_ARG;
    for (int h = 0; h < n; ++h) {
        if (!(sigmas[h] > 0)) return nb_fail(b, MTD_ERR_INVALID_ARG, "hill widths must be positive");
        double rec[8] = {0, 0, 0, 0, heights[h], 0.5 / (sigmas[h] * sigmas[h]), 1.0 / (sigmas[h] * sigmas[h]), 0};
        for (int k = 0; k < b->D; ++k) rec[k] = centers[(size_t)h * b->D + k];
        b->hills.insert(b->hills.end(), rec, rec + 8);
    }
    const int nh = (int)(b->hills.size() / 8);
    if (nh > b->cap_h) {
        if (b->d_hills) cudaFree(b->d_hills);
        b->d_hills = nullptr;
        const int cap = nh + nh / 2 + 64;
        NB_CU(cudaMalloc(&b->d_hills, sizeof(double) * 8 * (size_t)cap), "hills");
        b->cap_h = cap;
        NB_CU(cudaMemcpyAsync(b->d_hills, b->hills.data(), sizeof(double) * b->hills.size(), cudaMemcpyHostToDevice,
                              b->st),
              "hills");
    } else if (n > 0) {
        NB_CU(cudaMemcpyAsync(b->d_hills + (size_t)b->nh * 8, b->hills.data() + (size_t)b->nh * 8,
                              sizeof(double) * 8 * (size_t)n, cudaMemcpyHostToDevice, b->st),
              "hills");
    }
    b->nh = nh;
    b->validated = false;
    NB_CU(cudaStreamSynchronize(b->st), "hills");
    return MTD_OK;
}

int mtd_nnbias_num_hills(const mtd_nnbias *b) { return b ? b->nh : 0; }

mtd_status mtd_nnbias_exact(mtd_nnbias *b, int npts, const double *pts, double *V, double *dV) {
    if (!b || npts < 0 || (npts > 0 && (!pts || !V))) return MTD_ERR_INVALID_ARG;
    return nb_exact_host(b, npts, pts, V, dV);
}

mtd_status mtd_nnbias_eval(mtd_nnbias *b, int npts, const double *pts, double *V, double *dV) {
    if (!b || npts < 0 || (npts > 0 && (!pts || !V))) return MTD_ERR_INVALID_ARG;
    if (npts == 0) return MTD_OK;
    std::vector<float> x((size_t)npts * kIn);
    for (int i = 0; i < npts; ++i) nb_normalise(b, pts + (size_t)i * b->D, x.data() + (size_t)i * kIn);
    float *d_x = nullptr, *d_y = nullptr, *d_ds = nullptr;
    NB_CU(cudaMalloc(&d_x, sizeof(float) * x.size()), "points");
    NB_CU(cudaMalloc(&d_y, sizeof(float) * npts), "values");
    NB_CU(cudaMalloc(&d_ds, sizeof(float) * x.size()), "gradients");
    cudaMemcpyAsync(d_x, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice, b->st);
    mtd_status s = nb_forward_batch(b, npts, d_x, d_y, dV ? d_ds : nullptr);
    std::vector<float> y(npts), g(x.size());
    if (s == MTD_OK) {
        cudaMemcpyAsync(y.data(), d_y, sizeof(float) * npts, cudaMemcpyDeviceToHost, b->st);
        if (dV) cudaMemcpyAsync(g.data(), d_ds, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, b->st);
        s = nb_check_err(b);
    }
    cudaFree(d_x);
    cudaFree(d_y);
    cudaFree(d_ds);
    if (s != MTD_OK) return s;
    for (int i = 0; i < npts; ++i) {
        V[i] = b->vscale * (double)y[i];
        if (dV)
            for (int k = 0; k < b->D; ++k)
                dV[(size_t)i * b->D + k] = b->vscale * (double)g[(size_t)i * kIn + k] * 2.0 / (b->hi[k] - b->lo[k]);
    }
    return MTD_OK;
}

// One gradient of the MSE loss on given points and targets (no update): for
// checks against an independent implementation.  grad in the flat layout
// W1[128][4], b1, W2[128][128], b2, w3, b3 (17,281 values).
mtd_status mtd_nnbias_loss_grad(mtd_nnbias *b, int npts, const double *pts, const double *targets, double vscale,
                                float *grad, double *loss) {
    if (!b || npts <= 0 || !pts || !targets || !grad || !(vscale > 0)) return MTD_ERR_INVALID_ARG;
    std::vector<float> x((size_t)npts * kIn), t(npts);
    for (int i = 0; i < npts; ++i) {
        nb_normalise(b, pts + (size_t)i * b->D, x.data() + (size_t)i * kIn);
        t[i] = (float)(targets[i] / vscale);
    }
    const int ntiles = (npts + kH - 1) / kH;
    mtd_status s = nb_ensure_tiles(b, ntiles);
    if (s != MTD_OK) return s;
    s = nb_tile_attr(b);
    if (s != MTD_OK) return s;
    float *d_x = nullptr, *d_t = nullptr, *d_g = nullptr;
    NB_CU(cudaMalloc(&d_x, sizeof(float) * x.size()), "points");
    NB_CU(cudaMalloc(&d_t, sizeof(float) * npts), "targets");
    NB_CU(cudaMalloc(&d_g, sizeof(float) * kNPpad), "gradient");
    cudaMemcpyAsync(d_x, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice, b->st);
    cudaMemcpyAsync(d_t, t.data(), sizeof(float) * npts, cudaMemcpyHostToDevice, b->st);
    k_mlp_tile<MODE_TRAIN><<<ntiles, 128, kTileSmem, b->st>>>(nb_dev(b), npts, d_x, d_t, nullptr, nullptr, b->d_part,
                                                              b->d_loss, 2.0f / npts, b->d_err, b->wait_tries,
                                                              b->wait_stall);
    k_mlp_gradsum<<<(kNP + 255) / 256, 256, 0, b->st>>>(ntiles, b->d_part, d_g);
    std::vector<float> lp(ntiles);
    cudaMemcpyAsync(grad, d_g, sizeof(float) * kNP, cudaMemcpyDeviceToHost, b->st);
    cudaMemcpyAsync(lp.data(), b->d_loss, sizeof(float) * ntiles, cudaMemcpyDeviceToHost, b->st);
    s = nb_check_err(b);
    cudaFree(d_x);
    cudaFree(d_t);
    cudaFree(d_g);
    if (s != MTD_OK) return s;
    if (loss) {
        double l = 0.0;
        for (float v : lp) l += v;
        *loss = l / npts;
    }
    return MTD_OK;
}

mtd_status mtd_nnbias_get_params(mtd_nnbias *b, float *out) {
    if (!b || !out) return MTD_ERR_INVALID_ARG;
    NB_CU(cudaMemcpyAsync(out, b->d_master, sizeof(float) * kNP, cudaMemcpyDeviceToHost, b->st), "params");
    NB_CU(cudaStreamSynchronize(b->st), "params");
    return MTD_OK;
}

mtd_status mtd_nnbias_set_params(mtd_nnbias *b, const float *in, double vscale) {
    if (!b || !in || !(vscale > 0)) return MTD_ERR_INVALID_ARG;
    NB_CU(cudaMemcpyAsync(b->d_master, in, sizeof(float) * kNP, cudaMemcpyHostToDevice, b->st), "params");
    b->vscale = vscale;
    mtd_status s = nb_refresh_forward(b);
    if (s != MTD_OK) return s;
    NB_CU(cudaStreamSynchronize(b->st), "params");
    return MTD_OK;
}

double mtd_nnbias_vscale(const mtd_nnbias *b) { return b ? b->vscale : 0.0; }

// Fits the network to the hill sum: a pool of ntrain sampled points with
// exact FP64 targets, `iters` Adam steps on minibatches of `batch` points.
mtd_status mtd_nnbias_fit(mtd_nnbias *b, int ntrain, int iters, int batch, double lr, unsigned long long seed,
                          double *final_loss) {
    if (!b || ntrain < kH || iters < 0 || batch < kH || batch > ntrain || !(lr > 0)) return MTD_ERR_INVALID_ARG;
    if (b->nh == 0) return nb_fail(b, MTD_ERR_INVALID_ARG, "no hills to fit");
    std::vector<double> pts;
    nb_sample(b, ntrain, seed, pts);
    std::vector<double> V(ntrain);
    mtd_status s = nb_exact_host(b, ntrain, pts.data(), V.data(), nullptr);
    if (s != MTD_OK) return s;
    double vmax = 0.0;
    for (double v : V) vmax = std::max(vmax, std::fabs(v));
    const bool rescale = b->adam_t == 0 || vmax > 1.25 * b->vscale || vmax < 0.5 * b->vscale;
    if (rescale && vmax > 0) {   // output scale: refresh the last layer's scale with the data
        const double old = b->vscale;
        b->vscale = vmax;
        if (b->adam_t > 0 && old > 0) {
            std::vector<float> w(kNP);
            s = mtd_nnbias_get_params(b, w.data());
            if (s != MTD_OK) return s;
            const float f = (float)(old / vmax);
            for (int q = ow3; q < kNP; ++q) w[q] *= f;
            s = mtd_nnbias_set_params(b, w.data(), vmax);
            if (s != MTD_OK) return s;
        }
    }
    std::vector<float> x((size_t)ntrain * kIn), t(ntrain);
    for (int i = 0; i < ntrain; ++i) {
        nb_normalise(b, pts.data() + (size_t)i * b->D, x.data() + (size_t)i * kIn);
        t[i] = (float)(V[i] / b->vscale);
    }
    if (b->d_xt) cudaFree(b->d_xt);
    if (b->d_tt) cudaFree(b->d_tt);
    b->d_xt = nullptr;
    b->d_tt = nullptr;
    NB_CU(cudaMalloc(&b->d_xt, sizeof(float) * x.size()), "training points");
    NB_CU(cudaMalloc(&b->d_tt, sizeof(float) * ntrain), "training targets");
    cudaMemcpyAsync(b->d_xt, x.data(), sizeof(float) * x.size(), cudaMemcpyHostToDevice, b->st);
    cudaMemcpyAsync(b->d_tt, t.data(), sizeof(float) * ntrain, cudaMemcpyHostToDevice, b->st);
    b->ntrain = ntrain;
    const int ntiles = (batch + kH - 1) / kH;
    s = nb_ensure_tiles(b, ntiles);
    if (s != MTD_OK) return s;
    s = nb_tile_attr(b);
    if (s != MTD_OK) return s;
    const int nbatches = ntrain / batch;
    for (int it = 0; it < iters; ++it) {
        const int bi = it % nbatches;
        const int nb = batch;
        ++b->adam_t;
        const float b1c = 1.0f - std::pow(0.9f, (float)b->adam_t), b2c = 1.0f - std::pow(0.999f, (float)b->adam_t);
        const float lr_t = (float)(lr * (it < iters / 2 ? 1.0 : 0.5 * (1.0 + std::cos(M_PI * (it - iters / 2) /
                                                                                   std::max(1, iters - iters / 2)))));
        k_mlp_tile<MODE_TRAIN><<<ntiles, 128, kTileSmem, b->st>>>(
            nb_dev(b), nb, b->d_xt + (size_t)bi * batch * kIn, b->d_tt + (size_t)bi * batch, nullptr, nullptr,
            b->d_part, b->d_loss, 2.0f / nb, b->d_err, b->wait_tries, b->wait_stall);
        k_mlp_adam<<<(kNP + 255) / 256, 256, 0, b->st>>>(ntiles, b->d_part, b->d_master, b->d_mom, b->d_vel,
                                                         std::max(lr_t, (float)(lr * 0.02)), b1c, b2c, b->d_W1,
                                                         b->d_b1, b->d_W2, b->d_W2t, b->d_b2, b->d_w3, b->d_b3, 1);
    }
    NB_CU(cudaGetLastError(), "training");
    std::vector<float> lp(ntiles);
    cudaMemcpyAsync(lp.data(), b->d_loss, sizeof(float) * ntiles, cudaMemcpyDeviceToHost, b->st);
    s = nb_check_err(b);
    if (s != MTD_OK) return s;
    if (final_loss) {
        double l = 0.0;
        for (float v : lp) l += v;
        *final_loss = l / batch * b->vscale * b->vscale;
    }
    b->validated = false;
    return MTD_OK;
}

// Max and RMS of |V_theta - V_exact| on npts sampled points (the measure of the
// network's error); marks the network usable when max <= tol.
mtd_status mtd_nnbias_validate(mtd_nnbias *b, int npts, unsigned long long seed, double tol, double *max_err,
                               double *rms_err) {
    if (!b || npts <= 0) return MTD_ERR_INVALID_ARG;
    std::vector<double> pts;
    nb_sample(b, npts, seed, pts);
    std::vector<double> Ve(npts), Vn(npts);
    mtd_status s = nb_exact_host(b, npts, pts.data(), Ve.data(), nullptr);
    if (s != MTD_OK) return s;
    s = mtd_nnbias_eval(b, npts, pts.data(), Vn.data(), nullptr);
    if (s != MTD_OK) return s;
    double mx = 0.0, ss = 0.0;
    for (int i = 0; i < npts; ++i) {
        const double d = std::fabs(Vn[i] - Ve[i]);
        mx = std::max(mx, d);
        ss += d * d;
    }
    if (max_err) *max_err = mx;
    if (rms_err) *rms_err = std::sqrt(ss / npts);
    b->tol = tol;
    b->last_max_err = mx;
    b->validated = mx <= tol;
    return MTD_OK;
}

int mtd_nnbias_usable(const mtd_nnbias *b) { return b && b->validated ? 1 : 0; }

// Bias at one device-resident point (D doubles) into d_V (1) and d_dV (D),
// enqueued on `stream`: use_nn = 1 the network, 0 the exact hill sum,
// -1 the network when the last validation passed, else the exact sum.
mtd_status mtd_nnbias_eval_device(mtd_nnbias *b, int npts, const double *d_pts, double *d_V, double *d_dV,
                                  int use_nn, void *stream) {
    if (!b || npts < 0 || (npts > 0 && (!d_pts || !d_V))) return MTD_ERR_INVALID_ARG;
    if (npts == 0) return MTD_OK;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->st;
    const bool nn = use_nn > 0 || (use_nn < 0 && b->validated);
    const int nb = (npts + 255) / 256;
    if (!nn) {
        if (b->nh == 0) {
            NB_CU(cudaMemsetAsync(d_V, 0, sizeof(double) * npts, st), "bias");
            if (d_dV) NB_CU(cudaMemsetAsync(d_dV, 0, sizeof(double) * npts * b->D, st), "bias");
            return MTD_OK;
        }
        k_hillsum_batch<<<nb, 256, 0, st>>>(b->D, npts, d_pts, b->D, b->nh, b->d_hills, d_V, d_dV, b->D);
        NB_CU(cudaGetLastError(), "exact hill sum");
        return MTD_OK;
    }
    if (npts > b->cap_b) {
        cudaFree(b->d_bx);
        cudaFree(b->d_by);
        cudaFree(b->d_bds);
        b->d_bx = b->d_by = b->d_bds = nullptr;
        b->cap_b = 0;
        NB_CU(cudaMalloc(&b->d_bx, sizeof(float) * (size_t)npts * kIn), "points");
        NB_CU(cudaMalloc(&b->d_by, sizeof(float) * (size_t)npts), "values");
        NB_CU(cudaMalloc(&b->d_bds, sizeof(float) * (size_t)npts * kIn), "gradients");
        b->cap_b = npts;
    }
    double sc[kIn];
    for (int k = 0; k < kIn; ++k) sc[k] = 2.0 / (b->hi[k] - b->lo[k]);
    k_nb_inputs<<<nb, 256, 0, st>>>(b->D, npts, d_pts, b->lo[0], b->lo[1], b->lo[2], b->lo[3], sc[0], sc[1], sc[2],
                                    sc[3], b->d_bx);
    mtd_status s = nb_tile_attr(b);
    if (s != MTD_OK) return s;
    const int ntiles = (npts + kH - 1) / kH;
    if (d_dV)
        k_mlp_tile<MODE_GRAD_S><<<ntiles, 128, kTileSmem, st>>>(nb_dev(b), npts, b->d_bx, nullptr, b->d_by, b->d_bds,
                                                                nullptr, nullptr, 0.f, b->d_err, b->wait_tries,
                                                                b->wait_stall);
    else
        k_mlp_tile<MODE_FWD><<<ntiles, 128, kTileSmem, st>>>(nb_dev(b), npts, b->d_bx, nullptr, b->d_by, nullptr,
                                                             nullptr, nullptr, 0.f, b->d_err, b->wait_tries,
                                                             b->wait_stall);
    k_nb_outputs<<<nb, 256, 0, st>>>(b->D, npts, b->d_by, b->d_bds, b->vscale, sc[0], sc[1], sc[2], sc[3], d_V, d_dV);
    NB_CU(cudaGetLastError(), "network");
    return MTD_OK;
}

mtd_status mtd_nnbias_sync(mtd_nnbias *b) {
    if (!b) return MTD_ERR_INVALID_ARG;
    return nb_check_err(b);
}

mtd_status mtd_nnbias_set_wait(mtd_nnbias *b, int tries, int stall) {
    if (!b || tries < 0) return MTD_ERR_INVALID_ARG;
    b->wait_tries = tries > 0 ? tries : kWaitTries;
    b->wait_stall = stall ? 1 : 0;
    return MTD_OK;
}

mtd_status mtd_nnbias_point_device(mtd_nnbias *b, const double *d_s, double *d_V, double *d_dV, int use_nn,
                                   void *stream) {
    if (!b || !d_s || !d_V || !d_dV) return MTD_ERR_INVALID_ARG;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->st;
    const bool nn = use_nn > 0 || (use_nn < 0 && b->validated);
    if (nn) {
        double sc[kIn];
        for (int k = 0; k < kIn; ++k) sc[k] = 2.0 / (b->hi[k] - b->lo[k]);
        k_mlp_point<<<1, 128, 0, st>>>(nb_dev(b), d_s, b->lo[0], b->lo[1], b->lo[2], b->lo[3], sc[0], sc[1], sc[2],
                                       sc[3], b->vscale, d_V, d_dV);
    } else {
        if (b->nh == 0) {
            NB_CU(cudaMemsetAsync(d_V, 0, sizeof(double), st), "bias");
            NB_CU(cudaMemsetAsync(d_dV, 0, sizeof(double) * b->D, st), "bias");
            return MTD_OK;
        }
        k_hillsum_point<<<kPointBlocks, 256, 0, st>>>(b->D, d_s, 0, b->nh, b->d_hills, b->d_ppart, b->d_ticket, d_V,
                                                      d_dV, 0);
    }
    NB_CU(cudaGetLastError(), "bias at a point");
    return MTD_OK;
}

}  // extern "C"

namespace mtd {

mtd_status nnbias_enqueue_vdv(mtd_nnbias *b, const double *d_s, double *d_vdv, bool nn, int h_from,
                              cudaStream_t st) {
    double *d_V = d_vdv, *d_dV = d_vdv + 1;
    int h0 = 0;
    if (nn) {
        double sc[kIn];
        for (int k = 0; k < kIn; ++k) sc[k] = 2.0 / (b->hi[k] - b->lo[k]);
        k_mlp_point<<<1, 128, 0, st>>>(nb_dev(b), d_s, b->lo[0], b->lo[1], b->lo[2], b->lo[3], sc[0], sc[1], sc[2],
                                       sc[3], b->vscale, d_V, d_dV);
        h0 = std::max(0, std::min(h_from, b->nh));
    } else if (b->nh == 0 || h_from >= b->nh) {
        NB_CU(cudaMemsetAsync(d_vdv, 0, sizeof(double) * (1 + b->D), st), "bias");
    }
    if (h0 < b->nh)
        k_hillsum_point<<<kPointBlocks, 256, 0, st>>>(b->D, d_s, h0, b->nh, b->d_hills, b->d_ppart, b->d_ticket, d_V,
                                                      d_dV, nn ? 1 : 0);
    NB_CU(cudaGetLastError(), "bias at the CV point");
    return MTD_OK;
}

}  // namespace mtd
