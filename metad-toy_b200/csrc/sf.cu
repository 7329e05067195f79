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
constexpr int kSkAtoms = 8;        // atoms per thread of the mixed-precision force pass
// k-tiles (k-vectors per pass over the atoms): Q of the partial-sum pass (a
// register tile of 2Q sums per thread), QF of the mixed-precision force pass
// (a shared-memory table chunk).  Every k is summed in the same order
// whatever the tile, so every tile gives bitwise-identical results; the
// autotuner picks them (SkDev::qv, ::qf).

// Mixed precision, phase tables: the phase of k at x is split as
//   k.x = sum_d T_d[k][c_d] + k.delta,   T_d[k][c] = k_d (o_d + (c + 1/2) h_d) mod 2 pi,
// with c_d the table cell of x_d and |delta_d| <= h_d / 2 the FP32 offset from
// its centre.  The tables are formed and reduced in FP64 once per box; a pair
// then costs three shared-memory loads and FP32 arithmetic only.  A
// coordinate outside the tables' range takes the FP64 phase instead.
struct TabCell {
    int c[3];
    float dl[3];
    bool in;
};
__device__ __forceinline__ TabCell tab_cell(const SkDev &d, double x, double y, double z) {
    TabCell t;
    const double v[3] = {x, y, z};
    t.in = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double u = (v[a] - d.to[a]) * d.tih[a];
        const int c = (int)floor(u);
        t.in = t.in && u >= 0.0 && c < d.nct[a];
        t.c[a] = c;
        t.dl[a] = (float)(v[a] - (d.to[a] + (c + 0.5) * d.th[a]));
    }
    return t;
}

// Copies the tables of k-vectors k0 .. k0 + Q - 1 into shared memory:
// tc[(a * Q + q) * tstride + c].
template <int Q> __device__ __forceinline__ void load_tab_chunk(const SkDev &d, int k0, float *tc) {
    const int per = Q * d.tstride;
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) {
        const int a = e / per, r = e - a * per, q = r / d.tstride, c = r - q * d.tstride;
        tc[e] = k0 + q < d.K ? __ldg(d.tab + ((size_t)a * d.K + k0 + q) * d.tstride + c) : 0.f;
    }
}

template <int Q>
__device__ __forceinline__ float tab_phase(const float *tc, int tstride, int q, const TabCell &t, const float *kf) {
    const float base = tc[q * tstride + t.c[0]] + tc[(Q + q) * tstride + t.c[1]] + tc[(2 * Q + q) * tstride + t.c[2]];
    return base + fmaf(kf[0], t.dl[0], fmaf(kf[1], t.dl[1], kf[2] * t.dl[2]));
}


// k-vectors (and, in the force pass, rho) staged in dynamic shared memory
// sized to K, so a small K leaves room for more resident blocks.
template <bool FP64, int QV> __global__ void __launch_bounds__(256) k_sk_partial(SkDev d) {
    constexpr int kSkChunk = 2 * QV;   // reals per register tile
    constexpr int kSkQ = QV;
    pdl_entry();
    __shared__ double smem[kSkChunk * 32];
    extern __shared__ double kk[];   // 3K doubles; mixed: then 3K floats and a table chunk
    float *kf = reinterpret_cast<float *>(kk + 3 * d.K);
    float *tc = kf + 3 * d.K;
    for (int t = threadIdx.x; t < 3 * d.K; t += blockDim.x) {
        kk[t] = d.k[t];
        if (!FP64) kf[t] = (float)d.k[t];
    }
    __syncthreads();
    double cnt = 0.0;
    for (int k0 = 0; k0 < d.K; k0 += kSkChunk / 2) {
        if (!FP64) {
            load_tab_chunk<kSkQ>(d, k0, tc);
            __syncthreads();
        }
        double acc[kSkChunk];
        // mixed precision: a thread's few atoms (grid-stride, about n / (1184 * 256))
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
            TabCell tcell{};
            if (!FP64) tcell = tab_cell(d, x, y, z);
#pragma unroll
            for (int q = 0; q < kSkChunk / 2; ++q) {
                const int kq = k0 + q;
                if (kq < d.K) {
                    if (FP64) {
                        const double ph = kk[3 * kq] * x + kk[3 * kq + 1] * y + kk[3 * kq + 2] * z;
                        double s, c;
                        sincos(ph, &s, &c);
                        acc[2 * q] += c;
                        acc[2 * q + 1] += s;
                    } else {
                        float s, c;
                        if (tcell.in) {
                            sincos_f32_reduced(tab_phase<kSkQ>(tc, d.tstride, q, tcell, kf + 3 * kq), s, c);
                        } else {
                            const double ph = kk[3 * kq] * x + kk[3 * kq + 1] * y + kk[3 * kq + 2] * z;
                            phase_sincos_f32(ph, s, c);
                        }
                        facc[2 * q] += c;
                        facc[2 * q + 1] += s;
                    }
                }
            }
        }
        if (!FP64) {
#pragma unroll
            for (int t = 0; t < kSkChunk; ++t) acc[t] = facc[t];
        }
        block_sum<kSkChunk>(acc, smem);
        if (threadIdx.x == 0)
            for (int q = 0; q < kSkChunk / 2; ++q)
                if (k0 + q < d.K) {
                    d.partials[(size_t)blockIdx.x * (2 * d.K + 2) + 2 * (k0 + q)] = acc[2 * q];
                    d.partials[(size_t)blockIdx.x * (2 * d.K + 2) + 2 * (k0 + q) + 1] = acc[2 * q + 1];
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

template <bool FP64>
__global__ void __launch_bounds__(256) k_sk_force(SkDev d, const double *__restrict__ f_src, double *__restrict__ f_dst,
                                                  SysDev s, CellGrid g, double *vpart) {
    pdl_entry();
    __shared__ double smem[6 * 32];
    extern __shared__ double kk[];   // 3K doubles, then 2K doubles (FP64) or 5K floats (FP32)
    // FP64: rho as doubles; FP32: rho and k as floats (the per-atom gradient
    // is accumulated in FP32, the phase stays FP64)
    float *aux = reinterpret_cast<float *>(kk + 3 * d.K);
    double *rr = kk + 3 * d.K;
    float *rrf = aux, *kkf = aux + 2 * d.K;
    for (int t = threadIdx.x; t < 3 * d.K; t += blockDim.x) {
        kk[t] = d.k[t];
        if (!FP64) kkf[t] = (float)d.k[t];
    }
    for (int t = threadIdx.x; t < 2 * d.K; t += blockDim.x) {
        if (FP64) rr[t] = d.rho[t];
        else rrf[t] = (float)d.rho[t];
    }
    __syncthreads();
    const double a = d.coef[0];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double vir[6] = {0, 0, 0, 0, 0, 0};
    if (i < d.n) {
        double gx = 0, gy = 0, gz = 0;
        if (i < d.nown && (!d.mask || (d.mask[i] & d.groupbit))) {
            const double x = d.x[3 * i], y = d.x[3 * i + 1], z = d.x[3 * i + 2];
            if (FP64) {
                for (int q = 0; q < d.K; ++q) {
                    const double ph = kk[3 * q] * x + kk[3 * q + 1] * y + kk[3 * q + 2] * z;
                    double sn, cs;
                    sincos(ph, &sn, &cs);
                    const double w = -rr[2 * q] * sn + rr[2 * q + 1] * cs;
                    gx += w * kk[3 * q];
                    gy += w * kk[3 * q + 1];
                    gz += w * kk[3 * q + 2];
                }
            } else {
                float fx = 0.f, fy = 0.f, fz = 0.f;
                for (int q = 0; q < d.K; ++q) {
                    const double ph = kk[3 * q] * x + kk[3 * q + 1] * y + kk[3 * q + 2] * z;
                    float sn, cs;
                    phase_sincos_f32(ph, sn, cs);
                    const float w = fmaf(rrf[2 * q + 1], cs, -rrf[2 * q] * sn);
                    fx = fmaf(w, kkf[3 * q], fx);
                    fy = fmaf(w, kkf[3 * q + 1], fy);
                    fz = fmaf(w, kkf[3 * q + 2], fz);
                }
                gx = fx;
                gy = fy;
                gz = fz;
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

// Mixed precision force pass with the phase tables: each thread keeps the
// gradient of up to kSkAtoms atoms (grid stride) while the k-vectors pass by
// in chunks whose tables are staged in shared memory; the block's virial
// partial goes to vpart[blockIdx.x] and block 0 zeroes the partials of the
// one-atom-per-thread layout beyond the grid.
template <int kSkQF>
__global__ void __launch_bounds__(256) k_sk_force_tab(SkDev d, const double *__restrict__ f_src,
                                                      double *__restrict__ f_dst, SysDev s, CellGrid g,
                                                      double *vpart, int nparts) {
    pdl_entry();
    __shared__ double smem[6 * 32];
    extern __shared__ double kk[];   // 3K doubles, 3K floats (k), 2K floats (rho), the table chunk
    float *kf = reinterpret_cast<float *>(kk + 3 * d.K);
    float *rrf = kf + 3 * d.K;
    float *tc = rrf + 2 * d.K;
    for (int t = threadIdx.x; t < 3 * d.K; t += blockDim.x) {
        kk[t] = d.k[t];
        kf[t] = (float)d.k[t];
    }
    for (int t = threadIdx.x; t < 2 * d.K; t += blockDim.x) rrf[t] = (float)d.rho[t];
    const int stride = gridDim.x * blockDim.x;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    float fx[kSkAtoms], fy[kSkAtoms], fz[kSkAtoms];
#pragma unroll
    for (int j = 0; j < kSkAtoms; ++j) fx[j] = fy[j] = fz[j] = 0.f;
    for (int k0 = 0; k0 < d.K; k0 += kSkQF) {
        __syncthreads();
        load_tab_chunk<kSkQF>(d, k0, tc);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSkAtoms; ++j) {
            const int i = i0 + j * stride;
            if (i >= d.nown || (d.mask && !(d.mask[i] & d.groupbit))) continue;
            const double x = d.x[3 * i], y = d.x[3 * i + 1], z = d.x[3 * i + 2];
            const TabCell tcell = tab_cell(d, x, y, z);
            for (int q = 0; q < kSkQF && k0 + q < d.K; ++q) {
                const int kq = k0 + q;
                float sn, cs;
                if (tcell.in) {
                    sincos_f32_reduced(tab_phase<kSkQF>(tc, d.tstride, q, tcell, kf + 3 * kq), sn, cs);
                } else {
                    const double ph = kk[3 * kq] * x + kk[3 * kq + 1] * y + kk[3 * kq + 2] * z;
                    phase_sincos_f32(ph, sn, cs);
                }
                const float w = fmaf(rrf[2 * kq + 1], cs, -rrf[2 * kq] * sn);
                fx[j] = fmaf(w, kf[3 * kq], fx[j]);
                fy[j] = fmaf(w, kf[3 * kq + 1], fy[j]);
                fz[j] = fmaf(w, kf[3 * kq + 2], fz[j]);
            }
        }
    }
    const double a = d.coef[0];
    double vir[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < kSkAtoms; ++j) {
        const int i = i0 + j * stride;
        if (i >= d.n) continue;
        const double gx = -a * (double)fx[j], gy = -a * (double)fy[j], gz = -a * (double)fz[j];
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
        if (blockIdx.x == 0)
            for (int b = gridDim.x + threadIdx.x; b < nparts; b += blockDim.x)
                for (int t = 0; t < 6; ++t) vpart[(size_t)b * 8 + t] = 0.0;
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

// Dynamic shared memory above the 48 KB default (the phase-table chunks of a
// large K or a long box), granted once per kernel.
template <typename K> static void allow_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024)
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

size_t sk_table_smem(const SkDev &d, int q) { return sizeof(float) * 3 * q * (size_t)d.tstride; }

template <int QV> static void launch_sk_partial_mixed(const SkDev &d, cudaStream_t st) {
    const size_t sm = (sizeof(double) + sizeof(float)) * 3 * (size_t)d.K + sk_table_smem(d, QV);
    allow_smem(k_sk_partial<false, QV>, sm);
    launch_k(k_sk_partial<false, QV>, d.nblocks, 256, sm, st, d);
}

template <int QF>
static void launch_sk_force_mixed(const SkDev &d, const double *f_src, double *f_dst, const SysDev &s,
                                  const CellGrid &g, double *vpart, int nb, cudaStream_t st) {
    const int tb = (d.n + 256 * kSkAtoms - 1) / (256 * kSkAtoms);   // kSkAtoms atoms per thread
    const size_t sm = sizeof(double) * 3 * (size_t)d.K + sizeof(float) * 5 * (size_t)d.K + sk_table_smem(d, QF);
    allow_smem(k_sk_force_tab<QF>, sm);
    launch_k(k_sk_force_tab<QF>, tb, 256, sm, st, d, f_src, f_dst, s, g, vpart, nb);
}

size_t sk_smem_values(const SkDev &d, int qv) {
    return (sizeof(double) + sizeof(float)) * 3 * (size_t)d.K + sk_table_smem(d, qv);
}
size_t sk_smem_force(const SkDev &d, int qf) {
    return sizeof(double) * 3 * (size_t)d.K + sizeof(float) * 5 * (size_t)d.K + sk_table_smem(d, qf);
}

void launch_sk_values(const SkDev &d, cudaStream_t st) {
    if (d.fp64) {
        const size_t sm = sizeof(double) * 3 * (size_t)d.K;
        allow_smem(k_sk_partial<true, 8>, sm);
        launch_k(k_sk_partial<true, 8>, d.nblocks, 256, sm, st, d);
    } else if (d.qv == 4) {
        launch_sk_partial_mixed<4>(d, st);
    } else if (d.qv == 16) {
        launch_sk_partial_mixed<16>(d, st);
    } else {
        launch_sk_partial_mixed<8>(d, st);
    }
    prof_mark("sk_partial", st);
    launch_k(k_sk_reduce, 2 * d.K + 1, 256, 0, st, d);
    prof_mark("sk_reduce", st);
}

void launch_sk_forces(const SkDev &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                      double *vpart, cudaStream_t st) {
    if (d.n == 0) return;
    const int nb = (d.n + 255) / 256;
    if (d.fp64) {
        const size_t sm = sizeof(double) * 5 * (size_t)d.K;
        allow_smem(k_sk_force<true>, sm);
        launch_k(k_sk_force<true>, nb, 256, sm, st, d, f_src, f_dst, s, g, vpart);
    } else if (d.qf == 8) {
        launch_sk_force_mixed<8>(d, f_src, f_dst, s, g, vpart, nb, st);
    } else if (d.qf == 16) {
        launch_sk_force_mixed<16>(d, f_src, f_dst, s, g, vpart, nb, st);
    } else {
        launch_sk_force_mixed<32>(d, f_src, f_dst, s, g, vpart, nb, st);
    }
    prof_mark("sk_force", st);
}

}  // namespace mtd
