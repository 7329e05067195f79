// global_q.cu -- STEINH Q: per-atom q_lm / Q_l over the cap-N nearest
// neighbours, AVE and SW_FUNC reductions, and the exact analytic gradient.
//
// Replaces steinhardt_cv_kernel (src/cvs/CVs_Steinhardt.cu:1410-1532), the
// host reductions compute_cv_AVE / compute_cv_SW_FUNC (:825-839, :961-977) and
// the gradient kernels steinhardt_dcv_AVE_kernel / _SW_FUNC_kernel
// (:1538-1863).  The reference gradient drops the Re(q)dRe(Y) terms of odd m
// and the Im(q)dIm(Y) terms of even m >= 2 (include/CVsets/CV_Steinhardt_math.h
// :200-668) and weights SW_FUNC by (f + Q f') instead of f'; this kernel
// computes the exact derivative of the CV value the reference reports.
//
// Gather form: lam_i = dCV/dQ_i * 4 pi/(2l+1) / (Q_i n_i) * w_m q_im, and for
// atom a over the within-rc pairs (a, j):
//   Lam = [j kept by a] lam_a + [a kept by j] (-1)^l lam_j,
//   dCV/dx_a = - sum_j grad_d Re(Lam . Y(d_aj)).
// "a kept by j" is read from j's cap key (r2, caller index) of its last kept
// neighbour, so a binding cap is handled exactly.
#include "kernels.h"
#include "ylm.cuh"

#include <math_constants.h>

namespace mtd {

namespace {

template <int L> struct QSize {
    static constexpr int S = 2 * (L + 1);
    static constexpr int SQ = pad4(S);
};

template <int L, typename T> __global__ void __launch_bounds__(kBlock) k_global_values(GlobalDev<T> d) {
    pdl_entry();
    using Z = QSize<L>;
    __shared__ double smem[4 * 32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double part[4] = {0, 0, 0, 0};
    if (k < d.n) {
        const auto a = d.geo.load(k);
        const int c = min(d.nb.count[k], d.nb.M);
        T acc[Z::SQ];
#pragma unroll
        for (int t = 0; t < Z::SQ; ++t) acc[t] = T(0);
        int kept = 0;
        for (int t = 0; t < c; ++t) {
            const int e = d.nb.list[(size_t)t * d.npad + k];
            if (!((e >> kFlagBit) & 1)) continue;
            T dx, dy, dz;
            d.geo.disp(a, d.geo.load(e & ((1 << kFlagBit) - 1)), dx, dy, dz);
            const T rinv = t_rsqrt<T>(dx * dx + dy * dy + dz * dz);
            ylm_accum<L, T>(dx * rinv, dy * rinv, dz * rinv, T(1), acc);
            ++kept;
        }
        const T inv = kept > 0 ? T(1) / T(kept) : T(0);
#pragma unroll
        for (int t = 0; t < Z::SQ; ++t) acc[t] *= inv;
        T q2 = acc[0] * acc[0];
#pragma unroll
        for (int m = 1; m <= L; ++m) q2 += T(2) * (acc[2 * m] * acc[2 * m] + acc[2 * m + 1] * acc[2 * m + 1]);
        const T Q = kept > 0 ? t_sqrt<T>(q2 * T(4.0 * kPi / (2 * L + 1))) : T(0);
#pragma unroll
        for (int t = 0; t < Z::SQ; ++t) d.q[(size_t)k * Z::SQ + t] = acc[t];
        d.Q[k] = Q;
        if (d.smask[k] & d.groupbit) {
            part[0] = (double)Q;
            if (d.nsw > 0) part[1] = sw_f<double>(d.sw[0], (double)Q);
            if (d.nsw > 1) part[2] = sw_f<double>(d.sw[1], (double)Q);
            part[3] = 1.0;
        }
    }
    block_sum<4>(part, smem);
    if (threadIdx.x == 0)
        for (int t = 0; t < 4; ++t) d.partials[blockIdx.x * 8 + t] = part[t];
}

template <int L, typename T>
__device__ __forceinline__ T lambda_scale(const GlobalDev<T> &d, int k, const double *c) {
    if (!(d.smask[k] & d.groupbit)) return T(0);
    const int n = d.nb.nkept[k];
    const double Q = (double)d.Q[k];
    if (n <= 0 || !(Q > 0.0)) return T(0);
    double dcv = c[0];
    if (d.nsw > 0) dcv += c[1] * sw_df<double>(d.sw[0], Q);
    if (d.nsw > 1) dcv += c[2] * sw_df<double>(d.sw[1], Q);
    return (T)(dcv * (4.0 * kPi / (2 * L + 1)) / (Q * n));
}

template <int L, typename T>
__global__ void __launch_bounds__(kBlock) k_global_force(GlobalDev<T> d, const double *__restrict__ f_src,
                                                         double *__restrict__ f_dst, SysDev s, CellGrid g,
                                                         double *vpart, DevStatus *status) {
    pdl_entry();
    using Z = QSize<L>;
    __shared__ double smem[6 * 32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    const double c[3] = {d.coef[0], d.coef[1], d.coef[2]};
    if (k < d.n) {
        const T ak = lambda_scale<L, T>(d, k, c);
        T la[Z::SQ];
#pragma unroll
        for (int t = 0; t < Z::SQ; ++t) la[t] = ak * d.q[(size_t)k * Z::SQ + t] * (t >= 2 ? T(2) : T(1));
        const int myid = d.perm[k];
        const double xk[3] = {s.xs[3 * k], s.xs[3 * k + 1], s.xs[3 * k + 2]};
        const auto a = d.geo.load(k);
        constexpr T sgn = (L & 1) ? T(-1) : T(1);
        T gx = T(0), gy = T(0), gz = T(0);
        const int cnt = min(d.nb.count[k], d.nb.M);
        for (int t = 0; t < cnt; ++t) {
            const int e = d.nb.list[(size_t)t * d.npad + k];
            const bool kept = (e >> kFlagBit) & 1;
            const int j = e & ((1 << kFlagBit) - 1);
            bool rev = true;
            const double kr2 = d.nb.key_r2[j];
            if (kr2 != CUDART_INF) {
                const double xj[3] = {s.xs[3 * j], s.xs[3 * j + 1], s.xs[3 * j + 2]};
                double dd[3];
                const double r2 = exact_disp(d.exact, xj, xk, dd);
                rev = (r2 < kr2) || (r2 == kr2 && myid <= d.nb.key_id[j]);
            }
            const T aj = rev ? lambda_scale<L, T>(d, j, c) : T(0);
            if (!kept && aj == T(0)) continue;
            T Lm[Z::SQ];
#pragma unroll
            for (int q = 0; q < Z::SQ; ++q) {
                const T w = q >= 2 ? T(2) : T(1);
                Lm[q] = (kept ? la[q] : T(0)) + sgn * aj * w * d.q[(size_t)j * Z::SQ + q];
            }
            T dx, dy, dz;
            d.geo.disp(a, d.geo.load(j), dx, dy, dz);
            const T rinv = t_rsqrt<T>(dx * dx + dy * dy + dz * dz);
            T ax, ay, az;
            ylm_dot_grad<L, T>(dx * rinv, dy * rinv, dz * rinv, rinv, Lm, ax, ay, az);
            gx -= ax;
            gy -= ay;
            gz -= az;
        }
        const int i = myid;
        const double fx = -(double)gx, fy = -(double)gy, fz = -(double)gz;
        const bool own = (unsigned)i < (unsigned)d.n;   // a sorted order left by a rebuild that gave up is not trusted
        if (own) {
            f_dst[3 * i] = f_src[3 * i] + fx;
            f_dst[3 * i + 1] = f_src[3 * i + 1] + fy;
            f_dst[3 * i + 2] = f_src[3 * i + 2] + fz;
        }
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&status->nan_force, 1u);
        if (vpart && own) {
            double ux = xk[0], uy = xk[1], uz = xk[2];
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

}  // namespace

template <typename T> void launch_global_values(const GlobalDev<T> &d, cudaStream_t st) {
    if (d.n == 0) return;
    const int nb = (d.n + kBlock - 1) / kBlock;
    switch (d.L) {
    case 3: launch_k(k_global_values<3, T>, nb, kBlock, 0, st, d); break;
    case 4: launch_k(k_global_values<4, T>, nb, kBlock, 0, st, d); break;
    case 6: launch_k(k_global_values<6, T>, nb, kBlock, 0, st, d); break;
    }
    prof_mark("global_values", st);
}

template <typename T>
void launch_global_forces(const GlobalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s,
                          const CellGrid &g, double *vpart, DevStatus *status, cudaStream_t st) {
    if (d.n == 0) return;
    const int nb = (d.n + kBlock - 1) / kBlock;
    switch (d.L) {
    case 3: launch_k(k_global_force<3, T>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status); break;
    case 4: launch_k(k_global_force<4, T>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status); break;
    case 6: launch_k(k_global_force<6, T>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status); break;
    }
    prof_mark("global_force", st);
}

template void launch_global_values<float>(const GlobalDev<float> &, cudaStream_t);
template void launch_global_values<double>(const GlobalDev<double> &, cudaStream_t);
template void launch_global_forces<float>(const GlobalDev<float> &, const double *, double *, const SysDev &,
                                          const CellGrid &, double *, DevStatus *, cudaStream_t);
template void launch_global_forces<double>(const GlobalDev<double> &, const double *, double *, const SysDev &,
                                           const CellGrid &, double *, DevStatus *, cudaStream_t);

}  // namespace mtd
