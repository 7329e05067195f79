// common.cuh -- shared types, switching functions and small device helpers.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <type_traits>

namespace mtd {

constexpr double kPi = 3.14159265358979323846;
constexpr int kBlock = 256;          // threads per block for per-atom kernels
constexpr int kMaxSymbols = 16;      // SYMBOL entries per context
constexpr int kMaxDim = 4;           // CV_dim handled by the device grid kernel
constexpr int kFlagBit = 30;         // pair.j bit: neighbour kept by the centre (STEINH Q cap)

enum SwType { SW_LINE = 0, SW_STEP = 1, SW_FERMI = 2, SW_TANH = 3, SW_RATIONAL = 4 };

// Switching-function parameters passed by value to kernels; the same fields as
// SwitchFunctionRequest (include/utils/zqc_switch_function.h:24-31).
struct SwParams {
    int type;
    double r0, d0, alpha;
    int n, m;
};

template <typename T> __host__ __device__ __forceinline__ T ipow_t(T x, int n) {
    T r = T(1);
    T b = x;
    int e = n < 0 ? -n : n;
    while (e) {
        if (e & 1) r *= b;
        b *= b;
        e >>= 1;
    }
    return n < 0 ? T(1) / r : r;
}

template <typename T> __host__ __device__ __forceinline__ T t_exp(T x);
template <> __host__ __device__ __forceinline__ double t_exp<double>(double x) { return exp(x); }
template <> __host__ __device__ __forceinline__ float t_exp<float>(float x) { return expf(x); }
template <typename T> __host__ __device__ __forceinline__ T t_tanh(T x);
template <> __host__ __device__ __forceinline__ double t_tanh<double>(double x) { return tanh(x); }
template <> __host__ __device__ __forceinline__ float t_tanh<float>(float x) { return tanhf(x); }
template <typename T> __host__ __device__ __forceinline__ T t_sqrt(T x);
template <> __host__ __device__ __forceinline__ double t_sqrt<double>(double x) { return sqrt(x); }
template <> __host__ __device__ __forceinline__ float t_sqrt<float>(float x) { return sqrtf(x); }

// f and df of the switching functions, following
// include/utils/zqc_switch_function.h:163-313 case by case (the RATIONAL n == 2m
// branch returns 1 + x^m exactly as the reference does).
template <typename T> __host__ __device__ __forceinline__ T sw_f(const SwParams &p, T x) {
    switch (p.type) {
    case SW_LINE: return T(1);
    case SW_STEP: return (x < T(p.r0)) ? T(1) : T(0);
    case SW_FERMI: return T(1) / (T(1) + t_exp<T>(-T(p.alpha) * (x - T(p.r0))));
    case SW_TANH: return T(0.5) * (T(1) + t_tanh<T>(T(p.alpha) * (x - T(p.r0))));
    case SW_RATIONAL: {
        const int n = p.n, m = p.m;
        T y = (x - T(p.d0)) / T(p.r0);
        if (n == 6 && m == 12) { T y2 = y * y; T y6 = y2 * y2 * y2; return T(1) / (T(1) + y6); }
        if (n == 4 && m == 8) { T y2 = y * y; T y4 = y2 * y2; return T(1) / (T(1) + y4); }
        if (2 * n == m) return T(1) / (T(1) + ipow_t(y, n));
        if (n == 2 * m) return T(1) + ipow_t(y, m);
        return (T(1) - ipow_t(y, n)) / (T(1) - ipow_t(y, m));
    }
    default: return T(1);
    }
}

template <typename T> __host__ __device__ __forceinline__ T sw_df(const SwParams &p, T x) {
    switch (p.type) {
    case SW_LINE: return T(0);
    case SW_STEP: return T(0);
    case SW_FERMI: {
        T e = t_exp<T>(-T(p.alpha) * (x - T(p.r0)));
        T den = T(1) + e;
        return (T(p.alpha) * e) / (den * den);
    }
    case SW_TANH: {
        T t = t_tanh<T>(T(p.alpha) * (x - T(p.r0)));
        return T(0.5) * T(p.alpha) * (T(1) - t * t);
    }
    case SW_RATIONAL: {
        const int n = p.n, m = p.m;
        T y = (x - T(p.d0)) / T(p.r0);
        if (n == 6 && m == 12) {
            T y2 = y * y, y5 = y2 * y2 * y, y6 = y2 * y2 * y2;
            return -T(n) * y5 / ((T(1) + y6) * (T(1) + y6)) / T(p.r0);
        }
        if (n == 4 && m == 8) {
            T y2 = y * y, y3 = y2 * y, y4 = y2 * y2;
            return -T(n) * y3 / ((T(1) + y4) * (T(1) + y4)) / T(p.r0);
        }
        if (2 * n == m) {
            T a = ipow_t(y, n - 1), b = ipow_t(y, n);
            return -T(n) * a / ((T(1) + b) * (T(1) + b)) / T(p.r0);
        }
        if (n == 2 * m) return T(m) * ipow_t(y, m - 1) / T(p.r0);
        T ymm1 = ipow_t(y, m - 1), ym = ymm1 * y;
        T one_m = T(1) - ym;
        if ((one_m < T(0) ? -one_m : one_m) < T(1e-12)) return T(-0.5) * T(n * (n - m)) / T(m) / T(p.r0);
        T ynm1 = ipow_t(y, n - 1);
        return (T(n - m) * ynm1 * ym + T(m) * ymm1 - T(n) * ynm1) / (one_m * one_m) / T(p.r0);
    }
    default: return T(0);
    }
}

// Pair record of the neighbour lists: displacement x_j - x_i (minimum image,
// computed in FP64 and rounded to T) and the sorted index of j (bit kFlagBit
// marks a neighbour kept by the centre's cap).
template <typename T> struct alignas(16) Pair;
template <> struct alignas(16) Pair<float> { float x, y, z; int j; };
template <> struct alignas(16) Pair<double> { double x, y, z; int j; int pad; };

// Device-side error word shared by the kernels of one context.
struct DevStatus {
    unsigned int overflow;        // max neighbour count seen when above capacity
    unsigned int nan_force;       // a force component was not finite
    unsigned int timeout;         // a bounded wait gave up
    unsigned int bad_pos;         // an atom position was not finite (NaN or Inf)
    unsigned int cand_overflow;   // max skin-list candidate count seen when above capacity
    unsigned int pad[3];
};

// First statement of every step kernel: wait until the previous kernel of the
// stream has completed and its writes are visible, then let the next kernel's
// blocks be scheduled as this one's drain (no-ops without the PDL attribute).
__device__ __forceinline__ void pdl_entry() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// The two halves, for a kernel that does work before its wait.  A block of a
// kernel K starts only after every block of the previous kernel P has let
// dependents launch; when P let them launch after its own wait, P's
// predecessor (and everything before it) has completed and is visible.  So
// before its wait K may read what the kernel two places back (or earlier)
// wrote, and must not read what P writes.  A kernel that lets dependents
// launch before its wait gives its successor no such window: that successor
// must open with its wait.
__device__ __forceinline__ void pdl_release() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Deterministic block sum of up to NV doubles per thread (fixed shuffle tree,
// then warp 0 over the warp partials).  Result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *smem /* NV * 32 */) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int t = 0; t < NV; ++t) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[t] += __shfl_down_sync(0xffffffffu, v[t], o);
    }
    if (lane == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) smem[t * 32 + warp] = v[t];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int t = 0; t < NV; ++t) {
            double s = lane < nw ? smem[t * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
            v[t] = s;
        }
    }
}

// Warp sums of NV = 2^P doubles per lane, spread over the lanes: lane l ends
// with the sum of value l >> (5 - P).  Lanes 16, 8, ... apart swap the halves
// of their values each step (NV - 1 shuffles), then the remaining steps add
// whole sums.  Every value is summed over the same tree of lanes as
// block_sum's shuffle-down steps (pairs 16, 8, 4, 2, 1 apart; each addition
// has the same two operands, possibly swapped), so the sums are equal bit
// for bit.
template <int NV> struct Log2NV { static constexpr int v = NV <= 1 ? 0 : 1 + Log2NV<NV / 2>::v; };
template <> struct Log2NV<1> { static constexpr int v = 0; };

template <int NV> __device__ __forceinline__ double warp_sum_spread(double (&v)[NV], int lane) {
    constexpr int P = Log2NV<NV>::v;
    static_assert((1 << P) == NV && P <= 5, "NV: a power of two up to 32");
#pragma unroll
    for (int st = 0; st < P; ++st) {
        const int o = 16 >> st, h = (NV >> st) / 2;
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < h; ++j) {
            const double send = up ? v[j] : v[j + h];
            const double keep = up ? v[j + h] : v[j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    double r = v[0];
#pragma unroll
    for (int st = P; st < 5; ++st) r += __shfl_xor_sync(0xffffffffu, r, 16 >> st);
    return r;
}

// block_sum with the totals spread over warp 0 (lane l of warp 0 returns the
// total of value l >> (5 - P); other warps return 0): the same totals bit
// for bit, with NV - 1 + 5 - P shuffles per warp instead of 5 NV.
template <int NV> __device__ __forceinline__ double block_sum_spread(double (&v)[NV], double *smem /* NV * 32 */) {
    constexpr int P = Log2NV<NV>::v;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    const double r = warp_sum_spread<NV>(v, lane);
    if ((lane & ((32 >> P) - 1)) == 0) smem[(lane >> (5 - P)) * 32 + warp] = r;
    __syncthreads();
    double tot = 0.0;
    if (warp == 0) {
        double w[NV];
#pragma unroll
        for (int t = 0; t < NV; ++t) w[t] = lane < nw ? smem[t * 32 + lane] : 0.0;
        tot = warp_sum_spread<NV>(w, lane);
    }
    return tot;
}

}  // namespace mtd

namespace mtd {
template <typename T> __device__ __forceinline__ T t_rsqrt(T x);
template <> __device__ __forceinline__ float t_rsqrt<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double t_rsqrt<double>(double x) { return rsqrt(x); }

constexpr int pad4(int v) { return (v + 3) & ~3; }

// LAMMPS packed image flags (default 10-bit layout: IMGBITS 10, IMGMAX 512).
__device__ __forceinline__ void unpack_image(int img, int &ix, int &iy, int &iz) {
    ix = (img & 1023) - 512;
    iy = ((img >> 10) & 1023) - 512;
    iz = (img >> 20) - 512;
}
// sin and cos of pi * u for an FP64 phase u in half turns (the mixed-
// precision k-vector sums scale k by 1 / pi once, so u = (k / pi) . x):
// u is rounded to the nearest integer n in FP64 (adding 1.5 * 2^52 leaves n
// in the low mantissa bits, so no rounding or conversion instruction), the
// remainder f = u - n in [-1/2, 1/2] is exact in FP64 and goes to FP32,
// sin(pi f) = f P(f^2) and cos(pi f) = Q(f^2) come from polynomials of
// degree 4 and 5 in f^2, and (-1)^n flips both signs.  |u| < 2^51.
// P and Q are near-minimax on f in [0, 1/2]: least squares on Chebyshev
// nodes, reweighted toward equal error peaks (Lawson's algorithm), with
// maximum errors 6.7e-9 and 2.2e-10 in exact arithmetic, below the FP32
// rounding of the result (1.6e-7 with FP32 evaluation, the same as the
// degree-13 / degree-12 Taylor series they replace, two and one FMA fewer;
// fit_sincospi.py beside the library regenerates them).
constexpr float kSinP0 = (float)3.1415926402242746, kSinP1 = (float)-5.167710094404562,
                kSinP2 = (float)2.5500777409855013, kSinP3 = (float)-0.5982926899608115,
                kSinP4 = (float)0.07766048988359421;
constexpr float kCosQ0 = (float)0.9999999997811803, kCosQ1 = (float)-4.934802137317261,
                kCosQ2 = (float)4.058709167239208, kCosQ3 = (float)-1.3352120902337075,
                kCosQ4 = (float)0.23493771734282284, kCosQ5 = (float)-0.02439697684324065;
constexpr double kInvPi = 0.31830988618379067154;

// The sign flip of halfturn_sincos_f32 as a bit mask (bit 31 set for odd n),
// with sin(pi f) and cos(pi f) unsigned: callers that fold the sign into a
// later product take these three.
__device__ __forceinline__ unsigned halfturn_sincos_f32_parts(double u, float &s0, float &c0) {
    constexpr double kRound = 6755399441055744.0;   // 1.5 * 2^52
    const double t = u + kRound;
    const double f = u - (t - kRound);
    const float z = (float)f, z2 = z * z;
    float p = fmaf(z2, kSinP4, kSinP3);
    p = fmaf(p, z2, kSinP2);
    p = fmaf(p, z2, kSinP1);
    p = fmaf(p, z2, kSinP0);
    s0 = p * z;
    float q = fmaf(z2, kCosQ5, kCosQ4);
    q = fmaf(q, z2, kCosQ3);
    q = fmaf(q, z2, kCosQ2);
    q = fmaf(q, z2, kCosQ1);
    c0 = fmaf(q, z2, kCosQ0);
    return (unsigned)__double2loint(t) << 31;
}

__device__ __forceinline__ void halfturn_sincos_f32(double u, float &s, float &c) {
    float s0, c0;
    const unsigned sgn = halfturn_sincos_f32_parts(u, s0, c0);
    s = __uint_as_float(__float_as_uint(s0) ^ sgn);
    c = __uint_as_float(__float_as_uint(c0) ^ sgn);
}

// The same for a phase in radians (one FP64 multiply by 1 / pi first).
__device__ __forceinline__ void phase_sincos_f32(double ph, float &s, float &c) {
    halfturn_sincos_f32(ph * kInvPi, s, c);
}

}  // namespace mtd
