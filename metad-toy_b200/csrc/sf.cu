// sf.cu -- structure-factor CVs.
//
// STRU_FACTOR (Debye form) replaces structure_factor_cv_kernel and the AVE /
// COUNT gradient kernels (src/cvs/CVs_Strufactor.cu:1082-1271):
//   S_i = 1 + sum_{j: 1e-12 <= r2 <= rc2} sin(q r)/(q r) s(r),
//   s = 1 - ((r2 - 0.8 rc2)/(0.2 rc2))^3 above 0.8 rc2,
//   dCV/dx_a = - sum_j (a_a + a_j) g'(r_aj) dhat_aj,  a_i = dCV/dS_i.
// STRU_FACTOR_K (no reference counterpart): rho_k = sum_j exp(i k.x_j) over the
// group, S(k) = |rho_k|^2/N, CV = mean_k S(k),
//   dCV/dx_j = 2/(N K) sum_k k (-Re rho_k sin(k.x_j) + Im rho_k cos(k.x_j)).
// Phases are formed in FP64 and reduced to [-pi, pi] before an FP32 sincos;
// the sums over atoms are FP64 block partials reduced in a fixed order.
#include "kernels.h"

namespace mtd {

namespace {

template <typename T> __device__ __forceinline__ void t_sincos(T x, T *s, T *c);
template <> __device__ __forceinline__ void t_sincos<float>(float x, float *s, float *c) { sincosf(x, s, c); }
template <> __device__ __forceinline__ void t_sincos<double>(double x, double *s, double *c) { sincos(x, s, c); }

template <typename T> __device__ __forceinline__ void debye_g(T r2, T rc2, T qf, T &gv, T &dg) {
    const T r = t_sqrt<T>(r2), th = qf * r;
    T s = T(1), ds = T(0);
    const T r_on = T(0.8) * rc2;
    if (r2 > r_on) {
        const T t = (r2 - r_on) / (rc2 - r_on);
        s = T(1) - t * t * t;
        ds = T(-3) * t * t * (T(2) * r) / (rc2 - r_on);
    }
    if (qf == T(0)) {   // WEIGHT_CHEM: the taper alone is the pair term
        gv = s;
        dg = ds;
        return;
    }
    T sn, cs;
    t_sincos<T>(th, &sn, &cs);
    gv = sn / th * s;
    dg = (cs / th - sn / (th * th)) * s * qf + ds * sn / th;
}

// STRU_FACTOR Chemical: the type weight of every sorted atom (types outside
// the table weigh 0, as type 0 does).
template <typename T> __global__ void k_chem_weights(DebyeDev<T> d) {
    pdl_entry();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const int i = d.perm[k];
    const int t = (unsigned)i < (unsigned)d.n ? d.types[i] : 0;
    d.w[k] = (T)(t >= 0 && t < d.ntab ? d.wtab[t] : 0.0);
}

template <typename T> __global__ void __launch_bounds__(kBlock) k_debye_values(DebyeDev<T> d) {
    pdl_entry();
    __shared__ double smem[4 * 32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double part[4] = {0, 0, 0, 0};
    if (k < d.n) {
        T S = T(0);
        if (d.smask[k] & d.groupbit) {
            const int c = min(d.nb.count[k], d.nb.M);
            const T rc2 = (T)d.rc2, qf = (T)d.qf;
            const auto a = d.geo.load(k);
            const T wk = d.w ? d.w[k] : T(1);
            for (int t = 0; t < c; ++t) {
                const int j = d.nb.list[(size_t)t * d.npad + k];
                T dx, dy, dz;
                d.geo.disp(a, d.geo.load(j), dx, dy, dz);
                T gv, dg;
                debye_g<T>(dx * dx + dy * dy + dz * dz, rc2, qf, gv, dg);
                S += d.w ? wk * d.w[j] * gv : gv;
            }
            S += T(1);
            part[0] = (double)S;
            part[1] = sw_f<double>(d.sw, (double)S);
            part[2] = 1.0;
        }
        d.S[k] = S;
    }
    block_sum<4>(part, smem);
    if (threadIdx.x == 0)
        for (int t = 0; t < 4; ++t) d.partials[blockIdx.x * 8 + t] = part[t];
}

template <typename T>
__device__ __forceinline__ T debye_a(const DebyeDev<T> &d, int k, double c0, double c1) {
    if (!(d.smask[k] & d.groupbit)) return T(0);
    double a = c0;
    if (c1 != 0.0) a += c1 * sw_df<double>(d.sw, (double)d.S[k]);
    return (T)a;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_debye_force(DebyeDev<T> d, const double *__restrict__ f_src,
                                                        double *__restrict__ f_dst, SysDev s, CellGrid g,
                                                        double *vpart, DevStatus *status) {
    pdl_entry();
    __shared__ double smem[6 * 32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    const double c0 = d.coef[0], c1 = d.coef[1];
    if (k < d.n) {
        const T ak = debye_a<T>(d, k, c0, c1);
        const T rc2 = (T)d.rc2, qf = (T)d.qf;
        T gx = T(0), gy = T(0), gz = T(0);
        const int c = min(d.nb.count[k], d.nb.M);
        const auto a = d.geo.load(k);
        const T wk = d.w ? d.w[k] : T(1);
        for (int t = 0; t < c; ++t) {
            const int j = d.nb.list[(size_t)t * d.npad + k];
            T w = ak + debye_a<T>(d, j, c0, c1);
            if (d.w) w *= wk * d.w[j];
            if (w == T(0)) continue;
            T dx, dy, dz;
            d.geo.disp(a, d.geo.load(j), dx, dy, dz);
            const T r2 = dx * dx + dy * dy + dz * dz;
            T gv, dg;
            debye_g<T>(r2, rc2, qf, gv, dg);
            const T f = w * dg * t_rsqrt<T>(r2);
            gx -= f * dx;
            gy -= f * dy;
            gz -= f * dz;
        }
        const int i = d.perm[k];
        const double fx = -(double)gx, fy = -(double)gy, fz = -(double)gz;
        if ((unsigned)i < (unsigned)d.n) {   // a sorted order left by a rebuild that gave up is not trusted
            f_dst[3 * i] = f_src[3 * i] + fx;
            f_dst[3 * i + 1] = f_src[3 * i + 1] + fy;
            f_dst[3 * i + 2] = f_src[3 * i + 2] + fz;
        }
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&status->nan_force, 1u);
        if (vpart && (unsigned)i < (unsigned)d.n) {
            double ux = s.xs[3 * k], uy = s.xs[3 * k + 1], uz = s.xs[3 * k + 2];
            if (s.image) {
                int ix, iy, iz;
                unpack_image(s.image[i], ix, iy, iz);
                ux += ix * g.L[0];
                uy += iy * g.L[1];
                uz += iz * g.L[2];
            }
            vir[0] = fx * ux; vir[1] = fy * uy; vir[2] = fz * uz;
            vir[3] = fx * uy; vir[4] = fx * uz; vir[5] = fy * uz;
        }
    }
    if (vpart) {
        block_sum<6>(vir, smem);
        if (threadIdx.x == 0)
            for (int t = 0; t < 6; ++t) vpart[blockIdx.x * 8 + t] = vir[t];
    }
}

// ------------------------------------------------------------------ S(k)
constexpr int kSkBlocks = 148 * 4;  // grid for the partial sums (4 blocks per SM: more atoms per thread, fewer block sums)
// Shapes the autotuner picks (SkDev::qv, ::qf): QV k-vectors per pass over
// the atoms in the partial-sum pass (a register tile of 2 QV sums per thread),
// and the unroll depth U of the force pass's loop over k.  Every k is summed
// in the same order whatever the shape, so all give bitwise-identical
// results.  In mixed precision the phase (k / pi).x is formed in FP64 (B200
// runs FP64 at half the FP32 rate), reduced to half a turn in FP64 and
// finished with FP32 polynomials (halfturn_sincos_f32); a per-dimension FP32
// phase-table variant (three shared-memory loads and an FP32 reduction per
// pair) measured 2.2x slower and was removed.

template <bool FP64, int QV> __global__ void __launch_bounds__(256) k_sk_partial(SkDev d) {
    constexpr int kSkChunk = 2 * QV;   // reals per register tile
    pdl_entry();
    __shared__ double smem[kSkChunk * 32];
    extern __shared__ double kk[];   // 3K
    // mixed precision: k / pi, so the phases come out in half turns
    for (int t = threadIdx.x; t < 3 * d.K; t += blockDim.x) kk[t] = FP64 ? d.k[t] : d.k[t] * kInvPi;
    __syncthreads();
    double cnt = 0.0;
    for (int k0 = 0; k0 < d.K; k0 += QV) {
        double acc[kSkChunk];
        // mixed precision: a thread's few atoms (grid-stride, about n / (592 * 256))
        // are summed in FP32, every sum across threads and blocks in FP64
        float facc[kSkChunk];
#pragma unroll
        for (int t = 0; t < kSkChunk; ++t) {
            acc[t] = 0.0;
            facc[t] = 0.f;
        }
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < d.nown; i += gridDim.x * blockDim.x) {
            if (d.mask && !(d.mask[i] & d.groupbit)) continue;
            if (k0 == 0) cnt += 1.0;
            const double x = d.x[3 * i], y = d.x[3 * i + 1], z = d.x[3 * i + 2];
#pragma unroll
            for (int q = 0; q < QV; ++q) {
                const int kq = k0 + q;
                if (kq < d.K) {
                    const double ph = kk[3 * kq] * x + kk[3 * kq + 1] * y + kk[3 * kq + 2] * z;
                    if (FP64) {
                        double s, c;
                        sincos(ph, &s, &c);
                        acc[2 * q] += c;
                        acc[2 * q + 1] += s;
                    } else {
                        // the sign (-1)^n as a factor of exact FMAs: the same
                        // sums as adding the signed sin and cos
                        float s0, c0;
                        const unsigned sgn = halfturn_sincos_f32_parts(ph, s0, c0);
                        const float sg = __uint_as_float(0x3f800000u | sgn);
                        facc[2 * q] = fmaf(sg, c0, facc[2 * q]);
                        facc[2 * q + 1] = fmaf(sg, s0, facc[2 * q + 1]);
                    }
                }
            }
        }
        if (!FP64) {
#pragma unroll
            for (int t = 0; t < kSkChunk; ++t) acc[t] = facc[t];
        }
        // the chunk's 2 QV block totals land on the lanes of warp 0 (lane l:
        // value l >> (5 - log2(2 QV))), which write them side by side
        const double tot = block_sum_spread<kSkChunk>(acc, smem);
        constexpr int kSh = 5 - Log2NV<kSkChunk>::v;
        if (threadIdx.x < 32 && (threadIdx.x & ((1 << kSh) - 1)) == 0) {
            const int v = threadIdx.x >> kSh;
            if (k0 + (v >> 1) < d.K) d.partials[(size_t)blockIdx.x * (2 * d.K + 2) + 2 * k0 + v] = tot;
        }
        __syncthreads();
    }
    double c1[1] = {cnt};
    block_sum<1>(c1, smem);
    if (threadIdx.x == 0) d.partials[(size_t)blockIdx.x * (2 * d.K + 2) + 2 * d.K] = c1[0];
}

// One block per output value (2K rho components + the group count).
__global__ void __launch_bounds__(256) k_sk_reduce(SkDev d) {
    pdl_entry();
    __shared__ double smem[32];
    const int v = blockIdx.x;
    double acc[1] = {0.0};
    for (int b = threadIdx.x; b < d.nblocks; b += blockDim.x) acc[0] += d.partials[(size_t)b * (2 * d.K + 2) + v];
    block_sum<1>(acc, smem);
    if (threadIdx.x == 0) {
        if (v < 2 * d.K) d.rho[v] = acc[0];
        else *d.ngroup = acc[0];
    }
}

// FP64 force pass: one atom per thread, FP64 sincos of the FP64 phase.
template <int U>
__global__ void __launch_bounds__(256) k_sk_force(SkDev d, const double *__restrict__ f_src, double *__restrict__ f_dst,
                                                  SysDev s, CellGrid g, double *vpart) {
    pdl_entry();
    __shared__ double smem[6 * 32];
    extern __shared__ double kk[];   // 3K doubles of k, then 2K of rho
    double *rr = kk + 3 * d.K;
    for (int t = threadIdx.x; t < 3 * d.K; t += blockDim.x) kk[t] = d.k[t];
    for (int t = threadIdx.x; t < 2 * d.K; t += blockDim.x) rr[t] = d.rho[t];
    __syncthreads();
    const double a = d.coef[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    if (i < d.n) {
        double gx = 0, gy = 0, gz = 0;
        if (i < d.nown && (!d.mask || (d.mask[i] & d.groupbit))) {
            const double x = d.x[3 * i], y = d.x[3 * i + 1], z = d.x[3 * i + 2];
#pragma unroll U
            for (int q = 0; q < d.K; ++q) {
                const double ph = kk[3 * q] * x + kk[3 * q + 1] * y + kk[3 * q + 2] * z;
                double sn, cs;
                sincos(ph, &sn, &cs);
                const double w = -rr[2 * q] * sn + rr[2 * q + 1] * cs;
                gx += w * kk[3 * q];
                gy += w * kk[3 * q + 1];
                gz += w * kk[3 * q + 2];
            }
        }
        const double fx = -a * gx, fy = -a * gy, fz = -a * gz;
        f_dst[3 * i] = f_src[3 * i] + fx;
        f_dst[3 * i + 1] = f_src[3 * i + 1] + fy;
        f_dst[3 * i + 2] = f_src[3 * i + 2] + fz;
        if (vpart) {
            double ux = d.x[3 * i], uy = d.x[3 * i + 1], uz = d.x[3 * i + 2];
            if (s.image) {
                int ix, iy, iz;
                unpack_image(s.image[i], ix, iy, iz);
                ux += ix * g.L[0];
                uy += iy * g.L[1];
                uz += iz * g.L[2];
            }
            vir[0] = fx * ux; vir[1] = fy * uy; vir[2] = fz * uz;
            vir[3] = fx * uy; vir[4] = fx * uz; vir[5] = fy * uz;
        }
    }
    if (vpart) {
        block_sum<6>(vir, smem);
        if (threadIdx.x == 0)
            for (int t = 0; t < 6; ++t) vpart[blockIdx.x * 8 + t] = vir[t];
    }
}

// Mixed-precision force pass: AT atoms per thread (atoms blockIdx.x * 256 *
// AT + a * 256 + threadIdx.x), so each k's shared-memory loads serve AT
// atoms; per k one 16-byte load of (k / pi).xy, one of (Re rho, Im rho, kx,
// ky) in FP32 and two scalars.  Every atom sums its k terms in k order with
// the same operations whatever U and AT, so the shapes give identical forces.
template <int U, int AT>
__global__ void __launch_bounds__(256) k_sk_force_mixed(SkDev d, const double *__restrict__ f_src,
                                                        double *__restrict__ f_dst, SysDev s, CellGrid g,
                                                        double *vpart) {
    pdl_entry();
    __shared__ double smem[6 * 32];
    extern __shared__ double4 skf_raw[];   // K double2, K float4, K double, K float (44 K bytes)
    double2 *kxy = reinterpret_cast<double2 *>(skf_raw);
    float4 *rk = reinterpret_cast<float4 *>(kxy + d.K);
    double *kz = reinterpret_cast<double *>(rk + d.K);
    float *kzf = reinterpret_cast<float *>(kz + d.K);
    for (int q = threadIdx.x; q < d.K; q += blockDim.x) {
        kxy[q] = make_double2(d.k[3 * q] * kInvPi, d.k[3 * q + 1] * kInvPi);
        kz[q] = d.k[3 * q + 2] * kInvPi;
        rk[q] = make_float4((float)d.rho[2 * q], (float)d.rho[2 * q + 1], (float)d.k[3 * q], (float)d.k[3 * q + 1]);
        kzf[q] = (float)d.k[3 * q + 2];
    }
    __syncthreads();
    const double a = d.coef[0];
    double x[AT], y[AT], z[AT];
    float fx[AT], fy[AT], fz[AT];
    bool on[AT];
#pragma unroll
    for (int t = 0; t < AT; ++t) {
        const int i = (blockIdx.x * AT + t) * blockDim.x + threadIdx.x;
        on[t] = i < d.nown && (!d.mask || (d.mask[i] & d.groupbit));
        x[t] = on[t] ? d.x[3 * i] : 0.0;
        y[t] = on[t] ? d.x[3 * i + 1] : 0.0;
        z[t] = on[t] ? d.x[3 * i + 2] : 0.0;
        fx[t] = fy[t] = fz[t] = 0.f;
    }
    bool any = false;
#pragma unroll
    for (int t = 0; t < AT; ++t) any = any || on[t];
    if (any) {
#pragma unroll U
        for (int q = 0; q < d.K; ++q) {
            const double2 kq = kxy[q];
            const double kzq = kz[q];
            const float4 r = rk[q];
            const float kzq_f = kzf[q];
#pragma unroll
            for (int t = 0; t < AT; ++t) {
                const double u = kq.x * x[t] + kq.y * y[t] + kzq * z[t];
                float s0, c0;
                const unsigned sgn = halfturn_sincos_f32_parts(u, s0, c0);
                // Im rho cos - Re rho sin, with the sign (-1)^n applied after
                // (exact: rounding is symmetric in the sign)
                const float w = __uint_as_float(__float_as_uint(fmaf(r.y, c0, -r.x * s0)) ^ sgn);
                fx[t] = fmaf(w, r.z, fx[t]);
                fy[t] = fmaf(w, r.w, fy[t]);
                fz[t] = fmaf(w, kzq_f, fz[t]);
            }
        }
    }
    double vir[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int t = 0; t < AT; ++t) {
        const int i = (blockIdx.x * AT + t) * blockDim.x + threadIdx.x;
        if (i >= d.n) continue;
        const double gx = on[t] ? -a * (double)fx[t] : 0.0, gy = on[t] ? -a * (double)fy[t] : 0.0,
                     gz = on[t] ? -a * (double)fz[t] : 0.0;
        f_dst[3 * i] = f_src[3 * i] + gx;
        f_dst[3 * i + 1] = f_src[3 * i + 1] + gy;
        f_dst[3 * i + 2] = f_src[3 * i + 2] + gz;
        if (vpart) {
            double ux = d.x[3 * i], uy = d.x[3 * i + 1], uz = d.x[3 * i + 2];
            if (s.image) {
                int ix, iy, iz;
                unpack_image(s.image[i], ix, iy, iz);
                ux += ix * g.L[0];
                uy += iy * g.L[1];
                uz += iz * g.L[2];
            }
            vir[0] += gx * ux; vir[1] += gy * uy; vir[2] += gz * uz;
            vir[3] += gx * uy; vir[4] += gx * uz; vir[5] += gy * uz;
        }
    }
    if (vpart) {
        block_sum<6>(vir, smem);
        if (threadIdx.x == 0)
            for (int t = 0; t < 6; ++t) vpart[blockIdx.x * 8 + t] = vir[t];
    }
}

}  // namespace

template <typename T> void launch_debye_values(const DebyeDev<T> &d, cudaStream_t st) {
    if (d.n == 0) return;
    if (d.w) launch_k(k_chem_weights<T>, (d.n + kBlock - 1) / kBlock, kBlock, 0, st, d);
    launch_k(k_debye_values<T>, (d.n + kBlock - 1) / kBlock, kBlock, 0, st, d);
    prof_mark("debye_values", st);
}
template <typename T>
void launch_debye_forces(const DebyeDev<T> &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                         double *vpart, DevStatus *status, cudaStream_t st) {
    if (d.n == 0) return;
    launch_k(k_debye_force<T>, (d.n + kBlock - 1) / kBlock, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
    prof_mark("debye_force", st);
}
template void launch_debye_values<float>(const DebyeDev<float> &, cudaStream_t);
template void launch_debye_values<double>(const DebyeDev<double> &, cudaStream_t);
template void launch_debye_forces<float>(const DebyeDev<float> &, const double *, double *, const SysDev &,
                                         const CellGrid &, double *, DevStatus *, cudaStream_t);
template void launch_debye_forces<double>(const DebyeDev<double> &, const double *, double *, const SysDev &,
                                          const CellGrid &, double *, DevStatus *, cudaStream_t);

int sk_blocks(int n) {
    int b = (n + 255) / 256;
    return b < kSkBlocks ? (b < 1 ? 1 : b) : kSkBlocks;
}

template <int QV> static void launch_sk_partial_q(const SkDev &d, size_t sm, cudaStream_t st) {
    if (d.fp64) launch_k(k_sk_partial<true, QV>, d.nblocks, 256, sm, st, d);
    else launch_k(k_sk_partial<false, QV>, d.nblocks, 256, sm, st, d);
}

template <int U>
static void launch_sk_force_u(const SkDev &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                              double *vpart, size_t sm, int nb, cudaStream_t st) {
    if (d.fp64) {
        launch_k(k_sk_force<U>, nb, 256, sm, st, d, f_src, f_dst, s, g, vpart);
    } else if (vpart) {   // one atom per thread: one virial partial per 256 atoms, as the other units write
        launch_k(k_sk_force_mixed<U, 1>, nb, 256, sm, st, d, f_src, f_dst, s, g, vpart);
    } else {
        launch_k(k_sk_force_mixed<U, 2>, (d.n + 511) / 512, 256, sm, st, d, f_src, f_dst, s, g, vpart);
    }
}

void launch_sk_values(const SkDev &d, cudaStream_t st) {
    const size_t sm = sizeof(double) * 3 * (size_t)d.K;
    if (d.qv == 4) launch_sk_partial_q<4>(d, sm, st);
    else if (d.qv == 16) launch_sk_partial_q<16>(d, sm, st);
    else launch_sk_partial_q<8>(d, sm, st);
    prof_mark("sk_partial", st);
    launch_k(k_sk_reduce, 2 * d.K + 1, 256, 0, st, d);
    prof_mark("sk_reduce", st);
}

void launch_sk_forces(const SkDev &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                      double *vpart, cudaStream_t st) {
    if (d.n == 0) return;
    const int nb = (d.n + 255) / 256;
    const size_t sm = sizeof(double) * 3 * (size_t)d.K + (d.fp64 ? sizeof(double) * 2 : sizeof(float) * 5) * (size_t)d.K;
    if (d.qf == 1) launch_sk_force_u<1>(d, f_src, f_dst, s, g, vpart, sm, nb, st);
    else if (d.qf == 4) launch_sk_force_u<4>(d, f_src, f_dst, s, g, vpart, sm, nb, st);
    else launch_sk_force_u<2>(d, f_src, f_dst, s, g, vpart, sm, nb, st);
    prof_mark("sk_force", st);
}

}  // namespace mtd
