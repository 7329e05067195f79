// noalloc.cu -- k-vector structure factor with no device allocation.
//
// The same quantity as the STRU_FACTOR_K unit of a context,
//   rho(k) = sum_{i in group} exp(i k.x_i),   S = sum_k |rho(k)|^2 / (N K),
// computed from caller device buffers.  The block partial sums live in a
// file-scope device array of fixed size instead of memory from cudaMalloc, so
// a call allocates nothing: no cudaMalloc / cudaFree, no allocating library.
//
// Set-up: the first call on a device (that device current) looks up the
// array's address with cudaGetSymbolAddress and caches it.  That lookup can
// load the module, so make the first call before any stream capture.
//
// Scratch contents: every launch writes all the partial entries it later
// reads, so no part of the array has to start at zero.  Two calls in flight
// at the same time on one device share the array and race: order them on one
// stream (or with events).
#include <mutex>

#include "../../include/metad_b200.h"
#include "common.cuh"

namespace mtd {

namespace {

constexpr int kNaMaxK = 1024;                        // k-vectors per call
constexpr int kNaScratchDoubles = 1 << 17;           // 1 MiB of block partials
constexpr int kNaMaxBlocks = 148 * 4;                // partial-sum grid when the scratch allows
constexpr int kNaMaxDevices = 64;
constexpr int kNaChunk = 8;                          // reals per register tile (4 k-vectors)

static __device__ __align__(256) double g_na_scratch[kNaScratchDoubles];

// FP64: sincos of the FP64 phase.  Mixed: FP64 quadrant reduction, FP32
// series (phase_sincos_f32, the context's S(k) arithmetic).
template <bool FP64> __device__ __forceinline__ void na_sincos(double ph, double &s, double &c) {
    if (FP64) {
        sincos(ph, &s, &c);
    } else {
        float sf, cf;
        phase_sincos_f32(ph, sf, cf);
        s = sf;
        c = cf;
    }
}

// Block b writes scratch[b * (2K + 1) + v]: v < 2K the (Re, Im) rho partials,
// v = 2K the group count.
template <bool FP64>
__global__ void __launch_bounds__(256) k_na_partial(int n, const double *__restrict__ x, const int *__restrict__ mask,
                                                    int groupbit, int K, const double *__restrict__ kv,
                                                    double *__restrict__ scratch) {
    __shared__ double smem[kNaChunk * 32];
    __shared__ double kk[3 * kNaMaxK];
    for (int t = threadIdx.x; t < 3 * K; t += blockDim.x) kk[t] = kv[t];
    __syncthreads();
    const size_t row = (size_t)blockIdx.x * (2 * K + 1);
    double cnt = 0.0;
    for (int k0 = 0; k0 < K; k0 += kNaChunk / 2) {
        double acc[kNaChunk];
#pragma unroll
        for (int t = 0; t < kNaChunk; ++t) acc[t] = 0.0;
        const size_t stride = (size_t)gridDim.x * blockDim.x;
        for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < (size_t)n; i += stride) {
            if (mask && !(mask[i] & groupbit)) continue;
            if (k0 == 0) cnt += 1.0;
            const double px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
#pragma unroll
            for (int q = 0; q < kNaChunk / 2; ++q) {
                const int kq = k0 + q;
                if (kq < K) {
                    double s, c;
                    na_sincos<FP64>(kk[3 * kq] * px + kk[3 * kq + 1] * py + kk[3 * kq + 2] * pz, s, c);
                    acc[2 * q] += c;
                    acc[2 * q + 1] += s;
                }
            }
        }
        // block totals spread over warp 0 (lane l: value l / 4), as block_sum's
        const double tot = block_sum_spread<kNaChunk>(acc, smem);
        if (threadIdx.x < 32 && (threadIdx.x & 3) == 0 && k0 + (threadIdx.x >> 3) < K)
            scratch[row + 2 * k0 + (threadIdx.x >> 2)] = tot;
        __syncthreads();
    }
    double c1[1] = {cnt};
    block_sum<1>(c1, smem);
    if (threadIdx.x == 0) scratch[row + 2 * K] = c1[0];
}

// One block: every output summed over the blocks in block order, then S.
__global__ void __launch_bounds__(256) k_na_finish(int K, int nblocks, const double *__restrict__ scratch,
                                                   double *__restrict__ rho_out, double *__restrict__ s_out) {
    __shared__ double rho[2 * kNaMaxK + 1];
    for (int v = threadIdx.x; v < 2 * K + 1; v += blockDim.x) {
        double a = 0.0;
        for (int b = 0; b < nblocks; ++b) a += scratch[(size_t)b * (2 * K + 1) + v];
        rho[v] = a;
        if (rho_out && v < 2 * K) rho_out[v] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = 0.0;
        for (int k = 0; k < K; ++k) acc += rho[2 * k] * rho[2 * k] + rho[2 * k + 1] * rho[2 * k + 1];
        const double N = rho[2 * K];
        *s_out = N > 0.0 ? acc / N / K : 0.0;
    }
}

std::mutex g_na_mutex;
double *g_na_ptr[kNaMaxDevices] = {};

void na_msg(char *err, int errlen, const char *msg) {
    if (!err || errlen <= 0) return;
    int i = 0;
    for (; msg[i] && i < errlen - 1; ++i) err[i] = msg[i];
    err[i] = '\0';
}

}  // namespace

}  // namespace mtd

extern "C" mtd_status mtd_sk_noalloc(int n, const double *d_x, const int *d_mask, int groupbit, int nk,
                                     const double *d_k, int precision, double *d_rho, double *d_s, void *stream,
                                     char *err, int errlen) {
    using namespace mtd;
    na_msg(err, errlen, "");
    if (nk < 1 || nk > kNaMaxK) {
        na_msg(err, errlen, "mtd_sk_noalloc: nk must be in [1, 1024] (fixed scratch and shared-memory sizes)");
        return MTD_ERR_INVALID_ARG;
    }
    if (n < 0 || (n > 0 && !d_x)) {
        na_msg(err, errlen, "mtd_sk_noalloc: n must be >= 0 and d_x non-null when n > 0");
        return MTD_ERR_INVALID_ARG;
    }
    if (!d_k || !d_s) {
        na_msg(err, errlen, "mtd_sk_noalloc: d_k and d_s must be non-null device pointers");
        return MTD_ERR_INVALID_ARG;
    }
    if (precision != MTD_PREC_MIXED && precision != MTD_PREC_FP64) {
        na_msg(err, errlen, "mtd_sk_noalloc: precision must be MTD_PREC_MIXED or MTD_PREC_FP64");
        return MTD_ERR_INVALID_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        na_msg(err, errlen, "mtd_sk_noalloc: cudaGetDevice failed");
        return MTD_ERR_CUDA;
    }
    if (dev < 0 || dev >= kNaMaxDevices) {
        na_msg(err, errlen, "mtd_sk_noalloc: device ordinal beyond 63");
        return MTD_ERR_UNSUPPORTED;
    }
    double *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_na_mutex);
        if (!g_na_ptr[dev]) {   // set-up, once per device, with that device current
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_na_scratch);
            if (e != cudaSuccess || !p) {
                na_msg(err, errlen, "mtd_sk_noalloc: cudaGetSymbolAddress of the scratch array failed");
                return MTD_ERR_CUDA;
            }
            g_na_ptr[dev] = static_cast<double *>(p);
        }
        scratch = g_na_ptr[dev];
    }
    int nb = kNaScratchDoubles / (2 * nk + 1);
    if (nb > kNaMaxBlocks) nb = kNaMaxBlocks;
    const long long need = ((long long)n + 255) / 256;
    if (nb > need) nb = need > 0 ? (int)need : 1;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // each launch's own status (cudaGetLastError could report an earlier,
    // unrelated launch of the caller's as this call's failure)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nb);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaError_t e = precision == MTD_PREC_FP64
                        ? cudaLaunchKernelEx(&cfg, k_na_partial<true>, n, d_x, d_mask, groupbit, nk, d_k, scratch)
                        : cudaLaunchKernelEx(&cfg, k_na_partial<false>, n, d_x, d_mask, groupbit, nk, d_k, scratch);
    if (e == cudaSuccess) {
        cfg.gridDim = dim3(1);
        e = cudaLaunchKernelEx(&cfg, k_na_finish, nk, nb, (const double *)scratch, d_rho, d_s);
    }
    if (e != cudaSuccess) {
        na_msg(err, errlen, "mtd_sk_noalloc: kernel launch failed");
        return MTD_ERR_CUDA;
    }
    return MTD_OK;
}
