// local_body.cuh -- the STEINH L passes as per-thread bodies (one virtual
// block `bid` of blockDim.x sorted atoms each): record helpers, q_lm and NF,
// LQ_lm with the block partials, the adjoint lambda, and the gathered forces.
// Shared by the kernels of local_ql.cu and the persistent multi-walker step
// kernel.  The definitions are stated at the top of local_ql.cu.
#pragma once

#include "filter.cuh"
#include "ylm.cuh"

namespace mtd {

// Record layout: orders A then B, (Re, Im) per m; the stride is a multiple of
// 32 bytes so a record is read with 256-bit loads (8 floats or 4 doubles).
template <int LA, int LB, typename T> struct LSet {
    static constexpr int SA = 2 * (LA + 1);
    static constexpr int SB = LB ? 2 * (LB + 1) : 0;
    static constexpr int V32 = 32 / (int)sizeof(T);
    static constexpr int SQ = (SA + SB + V32 - 1) / V32 * V32;
};

// Reads a whole record with 32-byte vector loads (one L1 wavefront per 32
// bytes instead of per 16).  p must be 32-byte aligned: record strides are
// multiples of 32 bytes and the arrays come from cudaMalloc.
template <int N> __device__ __forceinline__ void load_rec32(const float *__restrict__ p, float (&v)[N]) {
    static_assert(N % 8 == 0, "record stride must be a multiple of 32 bytes");
#pragma unroll
    for (int i = 0; i < N / 8; ++i)
        asm("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=f"(v[8 * i]), "=f"(v[8 * i + 1]), "=f"(v[8 * i + 2]), "=f"(v[8 * i + 3]),
                       "=f"(v[8 * i + 4]), "=f"(v[8 * i + 5]), "=f"(v[8 * i + 6]), "=f"(v[8 * i + 7])
                     : "l"(p + 8 * i));
}
template <int N> __device__ __forceinline__ void load_rec32(const double *__restrict__ p, double (&v)[N]) {
    static_assert(N % 4 == 0, "record stride must be a multiple of 32 bytes");
#pragma unroll
    for (int i = 0; i < N / 4; ++i)
        asm("ld.global.nc.v4.f64 {%0,%1,%2,%3}, [%4];"
                     : "=d"(v[4 * i]), "=d"(v[4 * i + 1]), "=d"(v[4 * i + 2]), "=d"(v[4 * i + 3])
                     : "l"(p + 4 * i));
}

template <typename T, int N> __device__ __forceinline__ void load_rec(const T *__restrict__ p, T (&v)[N]) {
    static_assert(N % 4 == 0, "record stride");
    if constexpr (std::is_same<T, float>::value) {
        const float4 *q = reinterpret_cast<const float4 *>(p);
#pragma unroll
        for (int i = 0; i < N / 4; ++i) {
            float4 t = __ldg(q + i);
            v[4 * i] = t.x; v[4 * i + 1] = t.y; v[4 * i + 2] = t.z; v[4 * i + 3] = t.w;
        }
    } else {
        const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
        for (int i = 0; i < N / 2; ++i) {
            double2 t = __ldg(q + i);
            v[2 * i] = t.x; v[2 * i + 1] = t.y;
        }
    }
}

template <typename T, int N> __device__ __forceinline__ void store_rec(T *__restrict__ p, const T (&v)[N]) {
    if constexpr (std::is_same<T, float>::value) {
        float4 *q = reinterpret_cast<float4 *>(p);
#pragma unroll
        for (int i = 0; i < N / 4; ++i) q[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
    } else {
        double2 *q = reinterpret_cast<double2 *>(p);
#pragma unroll
        for (int i = 0; i < N / 2; ++i) q[i] = make_double2(v[2 * i], v[2 * i + 1]);
    }
}

// sum_m w_m |v_m|^2 with w_0 = 1, w_m = 2 (the reference's Q_l norm).
template <int L, typename T> __device__ __forceinline__ T qnorm2(const T *v) {
    T s = v[0] * v[0];
#pragma unroll
    for (int m = 1; m <= L; ++m) s += T(2) * (v[2 * m] * v[2 * m] + v[2 * m + 1] * v[2 * m + 1]);
    return s;
}

// Unit bond vector, 1/r, sigma and sigma' of a listed pair.
template <typename T, bool STEP>
__device__ __forceinline__ void pair_geom(const LocalDev<T> &d, const typename Geo<T>::Pos &a, int j, T &ux, T &uy,
                                          T &uz, T &rinv, T &sg, T &dsg) {
    T dx, dy, dz;
    d.geo.disp(a, d.geo.load(j), dx, dy, dz);
    const T r2 = dx * dx + dy * dy + dz * dz;
    rinv = t_rsqrt<T>(r2);
    ux = dx * rinv;
    uy = dy * rinv;
    uz = dz * rinv;
    if (STEP) {   // listed pairs of a STEP switch have sigma = 1 by construction
        sg = T(1);
        dsg = T(0);
    } else {
        const T r = r2 * rinv;
        sg = sw_f<T>(d.sw_r, r);
        dsg = sw_df<T>(d.sw_r, r);
    }
}

template <typename T, bool STEP>
__device__ __forceinline__ T pair_sigma(const LocalDev<T> &d, const typename Geo<T>::Pos &a, int j) {
    if (STEP) return T(1);
    T dx, dy, dz;
    d.geo.disp(a, d.geo.load(j), dx, dy, dz);
    return sw_f<T>(d.sw_r, t_sqrt<T>(dx * dx + dy * dy + dz * dz));
}

__device__ __forceinline__ int nb_index(const NeighDev &nb, int npad, int t, int k) {
    return __ldg(nb.list + (size_t)t * npad + k) & ((1 << kFlagBit) - 1);
}

// Pass 1: q_lm and NF for every atom.  With skin lists (FILTER) the pass
// first filters the atom's candidates into its exact list (the same
// decisions as k_filter), then sums over that list.
// With skin lists the pass filters the candidates first: in one loop with the
// sum (MERGED: the list is never read back) or in a filter loop followed by
// the sum over the exact list (no lane of a warp waits on another lane's
// Y_lm work during the filter).  Both sum in list order with the same
// operations, so they give identical results; the autotuner picks one.
template <int LA, int LB, typename T, bool STEP, bool FILTER, bool MERGED = true>
__device__ __forceinline__ void local_q_body(const LocalDev<T> &d, int bid) {
    using S = LSet<LA, LB, T>;
    const int k = bid * blockDim.x + threadIdx.x;
    if (FILTER && d.reset && k == 0) {
        SkinState *r = d.reset;
        if (r->gate) {
            r->age = 1;
            r->builds += 1;
        } else {
            r->age += 1;
        }
        r->gate = 0;
    }
    if (k >= d.n) return;
    const auto a = d.geo.load(k);
    T acc[S::SQ];
#pragma unroll
    for (int t = 0; t < S::SQ; ++t) acc[t] = T(0);
    T nf = T(0);
    int c = 0;
    if constexpr (FILTER && !MERGED) {
        constexpr int KIND = STEP ? NK_STEP : NK_SWITCH;
        const float4 af = __ldg(d.fgf.pf + k);
        const int nc = min(__ldg(d.cand.count + k), d.cand.M);
        int jn = nc > 0 ? __ldg(d.cand.list + k) : 0;
        float4 bn = nc > 0 ? __ldg(d.fgf.pf + jn) : make_float4(0.f, 0.f, 0.f, 0.f);
        int jn2 = nc > 1 ? __ldg(d.cand.list + (size_t)d.npad + k) : 0;
        for (int t = 0; t < nc; ++t) {
            const int j = jn;
            const float4 b = bn;
            if (t + 1 < nc) {
                jn = jn2;
                bn = __ldg(d.fgf.pf + jn);
            }
            if (t + 2 < nc) jn2 = __ldg(d.cand.list + (size_t)(t + 2) * d.npad + k);
            float fx, fy, fz;
            disp_f(d.fgf, af, b, fx, fy, fz);
            if (!decide<KIND>(d.fgd, d.fspec, d.fgd.xs, k, j, fx * fx + fy * fy + fz * fz)) continue;
            if (c < d.nb.M) d.nb.list[(size_t)c * d.npad + k] = j;
            ++c;
        }
        d.nb.count[k] = c;
        if (c > d.nb.M) atomicMax(&d.status->overflow, (unsigned)c);
        c = min(c, d.nb.M);
        // the sum over the list just written (this thread's own entries,
        // read back through the coherent path), index one iteration ahead
        int jl = c > 0 ? d.nb.list[k] : 0;
        for (int t = 0; t < c; ++t) {
            T ux, uy, uz, rinv, sg, dsg;
            const int j = jl;
            if (t + 1 < c) jl = d.nb.list[(size_t)(t + 1) * d.npad + k];
            pair_geom<T, STEP>(d, a, j, ux, uy, uz, rinv, sg, dsg);
            nf += sg;
            ylm_accum<LA, T>(ux, uy, uz, sg, acc);
            if constexpr (LB > 0) ylm_accum<LB, T>(ux, uy, uz, sg, acc + S::SA);
        }
    } else if constexpr (FILTER) {
        // one loop: each candidate is tested (the decisions of filter_atom)
        // and, when kept, written to the exact list and summed at once, so
        // the list is not read back; the sum runs in list order
        constexpr int KIND = STEP ? NK_STEP : NK_SWITCH;
        const float4 af = __ldg(d.fgf.pf + k);
        const int nc = min(__ldg(d.cand.count + k), d.cand.M);
        // the next candidate's position and the one after's index in flight,
        // so no load waits on another issued in the same iteration
        int jn = nc > 0 ? __ldg(d.cand.list + k) : 0;
        float4 bn = nc > 0 ? __ldg(d.fgf.pf + jn) : make_float4(0.f, 0.f, 0.f, 0.f);
        int jn2 = nc > 1 ? __ldg(d.cand.list + (size_t)d.npad + k) : 0;
        for (int t = 0; t < nc; ++t) {
            const int j = jn;
            const float4 b = bn;
            if (t + 1 < nc) {
                jn = jn2;
                bn = __ldg(d.fgf.pf + jn);
            }
            if (t + 2 < nc) jn2 = __ldg(d.cand.list + (size_t)(t + 2) * d.npad + k);
            float fx, fy, fz;
            disp_f(d.fgf, af, b, fx, fy, fz);
            if (!decide<KIND>(d.fgd, d.fspec, d.fgd.xs, k, j, fx * fx + fy * fy + fz * fz)) continue;
            if (c < d.nb.M) {
                d.nb.list[(size_t)c * d.npad + k] = j;
                T dx, dy, dz;
                if constexpr (sizeof(T) == sizeof(float)) {   // the same FP32 displacement pair_geom forms
                    dx = fx;
                    dy = fy;
                    dz = fz;
                } else {
                    d.geo.disp(a, d.geo.load(j), dx, dy, dz);
                }
                const T r2 = dx * dx + dy * dy + dz * dz;
                const T rinv = t_rsqrt<T>(r2);
                T sg = T(1);
                if (!STEP) sg = sw_f<T>(d.sw_r, r2 * rinv);
                nf += sg;
                ylm_accum<LA, T>(dx * rinv, dy * rinv, dz * rinv, sg, acc);
                if constexpr (LB > 0) ylm_accum<LB, T>(dx * rinv, dy * rinv, dz * rinv, sg, acc + S::SA);
            }
            ++c;
        }
        d.nb.count[k] = c;
        if (c > d.nb.M) atomicMax(&d.status->overflow, (unsigned)c);
        c = min(c, d.nb.M);
    } else {
        c = min(d.nb.count[k], d.nb.M);
        // each neighbour's index is loaded an iteration ahead, so its record
        // load waits on one memory latency instead of two
        int jn = c > 0 ? nb_index(d.nb, d.npad, 0, k) : 0;
        for (int t = 0; t < c; ++t) {
            T ux, uy, uz, rinv, sg, dsg;
            const int j = jn;
            if (t + 1 < c) jn = nb_index(d.nb, d.npad, t + 1, k);
            pair_geom<T, STEP>(d, a, j, ux, uy, uz, rinv, sg, dsg);
            nf += sg;
            ylm_accum<LA, T>(ux, uy, uz, sg, acc);
            if constexpr (LB > 0) ylm_accum<LB, T>(ux, uy, uz, sg, acc + S::SA);
        }
    }
    const bool active = c > 0 && nf >= T(1e-12);
    const T inv = active ? T(1) / nf : T(0);
#pragma unroll
    for (int t = 0; t < S::SQ; ++t) acc[t] *= inv;
    store_rec(d.q + (size_t)k * S::SQ, acc);
    d.nf[k] = active ? nf : T(0);
}

// Pass 2: LQ_lm, LQ, the e1/e2 weights of the adjoint and block partial sums.
template <int LA, int LB, typename T, bool STEP>
__device__ __forceinline__ void local_lq_body(const LocalDev<T> &d, int bid) {
    using S = LSet<LA, LB, T>;
    __shared__ double smem[8 * 32];
    const int k = bid * blockDim.x + threadIdx.x;
    const bool valid = k < d.n;
    double part[5] = {0, 0, 0, 0, 0};
    if (valid) {
        const bool ing = (d.smask[k] & d.groupbit) != 0;
        const T nfk = d.nf[k];
        T A[S::SQ];
        T lqA = T(0), lqB = T(0);
        if (ing && nfk > T(0)) {
            load_rec32(d.q + (size_t)k * S::SQ, A);
            const auto a = d.geo.load(k);
            const int c = min(d.nb.count[k], d.nb.M);
            // each neighbour's index is loaded an iteration ahead, so its record
            // load waits on one memory latency instead of two
            int jn = c > 0 ? nb_index(d.nb, d.npad, 0, k) : 0;
            for (int t = 0; t < c; ++t) {
                const int j = jn;
                if (t + 1 < c) jn = nb_index(d.nb, d.npad, t + 1, k);
                const T sg = pair_sigma<T, STEP>(d, a, j);
                T qj[S::SQ];
                load_rec32(d.q + (size_t)j * S::SQ, qj);
#pragma unroll
                for (int s = 0; s < S::SQ; ++s) A[s] += sg * qj[s];
            }
            const T inv = T(1) / (nfk + T(1));
#pragma unroll
            for (int s = 0; s < S::SQ; ++s) A[s] *= inv;
            lqA = t_sqrt<T>(qnorm2<LA, T>(A) * T(4.0 * kPi / (2 * LA + 1)));
            if constexpr (LB > 0) lqB = t_sqrt<T>(qnorm2<LB, T>(A + S::SA) * T(4.0 * kPi / (2 * LB + 1)));
        } else {
#pragma unroll
            for (int s = 0; s < S::SQ; ++s) A[s] = T(0);
        }
        d.lqs[2 * k] = lqA;
        d.lqs[2 * k + 1] = lqB;
        T e[4] = {T(0), T(0), T(0), T(0)};
        if (ing) {
            const double fA = sw_f<double>(d.sw_cvA, (double)lqA);
            part[0] = (double)lqA * fA;
            part[1] = fA;
            part[4] = 1.0;
            if (nfk > T(0)) {
                const double dfA = sw_df<double>(d.sw_cvA, (double)lqA);
                const double den = fmax((double)lqA, 1e-12) * ((double)nfk + 1.0);
                const double C = 4.0 * kPi / (2 * LA + 1);
                e[0] = (T)((dfA * lqA + fA) * C / den);
                e[1] = (T)(dfA * C / den);
            }
            if constexpr (LB > 0) {
                const double fB = sw_f<double>(d.sw_cvB, (double)lqB);
                part[2] = (double)lqB * fB;
                part[3] = fB;
                if (nfk > T(0)) {
                    const double dfB = sw_df<double>(d.sw_cvB, (double)lqB);
                    const double den = fmax((double)lqB, 1e-12) * ((double)nfk + 1.0);
                    const double C = 4.0 * kPi / (2 * LB + 1);
                    e[2] = (T)((dfB * lqB + fB) * C / den);
                    e[3] = (T)(dfB * C / den);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 4; ++t) d.e12[4 * k + t] = e[t];
        // the record's m = 0 imaginary slots (zero for LQ_l0, read by no
        // one as LQ) carry e1 of each order, so the lambda pass gathers one
        // record per neighbour instead of two
        A[1] = e[0];
        if constexpr (LB > 0) A[S::SA + 1] = e[2];
        store_rec(d.lq + (size_t)k * S::SQ, A);
    }
    // the five totals (padded to eight) spread over warp 0, lane l holding
    // value l / 4: the same sums as block_sum's, with fewer shuffles
    double p8[8] = {part[0], part[1], part[2], part[3], part[4], 0.0, 0.0, 0.0};
    const double tot = block_sum_spread<8>(p8, smem);
    if (threadIdx.x < 20 && (threadIdx.x & 3) == 0) d.partials[bid * 8 + (threadIdx.x >> 2)] = tot;
}

// G = (c1 e1 + c2 e2) w_m LQ_lm for one order, accumulated with weight s.
template <int L, typename T>
__device__ __forceinline__ void add_g(T *acc, const T *lq, T w, T s) {
    const T a = s * w;
    acc[0] += a * lq[0];
#pragma unroll
    for (int m = 1; m <= L; ++m) {
        acc[2 * m] += T(2) * a * lq[2 * m];
        acc[2 * m + 1] += T(2) * a * lq[2 * m + 1];
    }
}

// A CV switch whose derivative is identically zero (e2 = 0 for every atom).
__device__ __forceinline__ bool sw_flat(const SwParams &p) { return p.type == SW_LINE || p.type == SW_STEP; }

// Pass 3 for a step pair switch and flat CV switches: with e2 = 0 the weight
// of an order is c1 e1, so lam_k = c1 / NF_k * (e1_k LQ_k + sum_j s_kj e1_j
// LQ_j), and the sum needs no coefficient.  It is formed before `pdl` waits
// for the bias kernel (which writes the coefficients; e1 and LQ come from the
// LQ pass before it), so the gather of the first wave of blocks overlaps the
// bias kernel's serial phases.
template <int LA, int LB, typename T>
__device__ __forceinline__ void local_lambda_e1_body(const LocalDev<T> &d, int bid, bool pdl) {
    using S = LSet<LA, LB, T>;
    if (pdl) pdl_release();
    const int k = bid * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const T nfk = d.nf[k];
    T acc[S::SQ];
#pragma unroll
    for (int s = 0; s < S::SQ; ++s) acc[s] = T(0);
    if (!(nfk > T(0))) {
        store_rec(d.lam + (size_t)k * S::SQ, acc);
        return;
    }
    // e1 of each order travels in the LQ record's m = 0 imaginary slot
    // (written by the LQ pass), so each neighbour costs one record gather
    T lqk[S::SQ];
    load_rec32(d.lq + (size_t)k * S::SQ, lqk);
    add_g<LA, T>(acc, lqk, lqk[1], T(1));
    if constexpr (LB > 0) add_g<LB, T>(acc + S::SA, lqk + S::SA, lqk[S::SA + 1], T(1));
    const auto a = d.geo.load(k);
    const int c = min(d.nb.count[k], d.nb.M);
    int jn = c > 0 ? nb_index(d.nb, d.npad, 0, k) : 0;
    for (int t = 0; t < c; ++t) {
        const int j = jn;
        if (t + 1 < c) jn = nb_index(d.nb, d.npad, t + 1, k);
        T lqj[S::SQ];
        load_rec32(d.lq + (size_t)j * S::SQ, lqj);
        const T e1A = lqj[1], e1B = LB > 0 ? lqj[S::SA + 1] : T(0);
        if (e1A == T(0) && e1B == T(0)) continue;
        const T sg = pair_sigma<T, true>(d, a, j);
        add_g<LA, T>(acc, lqj, e1A, sg);
        if constexpr (LB > 0) add_g<LB, T>(acc + S::SA, lqj + S::SA, e1B, sg);
    }
    if (pdl) pdl_wait();
    const T inv = T(1) / nfk;
    const T sA = (T)d.coef[0] * inv, sB = (T)d.coef[2] * inv;
#pragma unroll
    for (int s = 0; s < S::SA; ++s) acc[s] *= sA;
#pragma unroll
    for (int s = S::SA; s < S::SQ; ++s) acc[s] *= sB;
    store_rec(d.lam + (size_t)k * S::SQ, acc);
}

// Pass 3 (after the bias kernel): lam_k / NF_k, and for smooth switches G_k,
// t_k, u_k.  `pdl`: the kernel was launched as a dependent launch and the
// body places its wait (the walker kernel passes false).
template <int LA, int LB, typename T, bool STEP>
__device__ __forceinline__ void local_lambda_body(const LocalDev<T> &d, int bid, bool pdl = false) {
    using S = LSet<LA, LB, T>;
    constexpr bool DSIG = !STEP;
    if constexpr (STEP) {
        if (sw_flat(d.sw_cvA) && (LB == 0 || sw_flat(d.sw_cvB))) {
            local_lambda_e1_body<LA, LB, T>(d, bid, pdl);
            return;
        }
    }
    if (pdl) pdl_entry();
    const int k = bid * blockDim.x + threadIdx.x;
    if (k >= d.n) return;
    const T c1A = (T)d.coef[0], c2A = (T)d.coef[1], c1B = (T)d.coef[2], c2B = (T)d.coef[3];
    const T nfk = d.nf[k];
    T lam[S::SQ];
#pragma unroll
    for (int s = 0; s < S::SQ; ++s) lam[s] = T(0);
    if (!(nfk > T(0))) {
        store_rec(d.lam + (size_t)k * S::SQ, lam);
        if constexpr (DSIG) {
            store_rec(d.g + (size_t)k * S::SQ, lam);
#pragma unroll
            for (int t = 0; t < 4; ++t) d.tu[4 * k + t] = T(0);
        }
        return;
    }
    T lqk[S::SQ];
    load_rec32(d.lq + (size_t)k * S::SQ, lqk);
    const T wA = c1A * d.e12[4 * k] + c2A * d.e12[4 * k + 1];
    const T wB = c1B * d.e12[4 * k + 2] + c2B * d.e12[4 * k + 3];
    add_g<LA, T>(lam, lqk, wA, T(1));
    if constexpr (LB > 0) add_g<LB, T>(lam + S::SA, lqk + S::SA, wB, T(1));
    T Gk[S::SQ];
    if constexpr (DSIG) {
#pragma unroll
        for (int s = 0; s < S::SQ; ++s) Gk[s] = lam[s];
    }
    const auto a = d.geo.load(k);
    const int c = min(d.nb.count[k], d.nb.M);
    // each neighbour's index is loaded an iteration ahead, so its record
    // load waits on one memory latency instead of two
    int jn = c > 0 ? nb_index(d.nb, d.npad, 0, k) : 0;
    for (int t = 0; t < c; ++t) {
        const int j = jn;
        if (t + 1 < c) jn = nb_index(d.nb, d.npad, t + 1, k);
        T ej[4];
        load_rec(d.e12 + 4 * (size_t)j, ej);
        // the record is loaded beside the weights, not after the test on them
        // (a zero weight is rare), so the two loads share one latency
        T lqj[S::SQ];
        load_rec32(d.lq + (size_t)j * S::SQ, lqj);
        const T wjA = c1A * ej[0] + c2A * ej[1];
        const T wjB = c1B * ej[2] + c2B * ej[3];
        if (wjA == T(0) && wjB == T(0)) continue;
        const T sg = pair_sigma<T, STEP>(d, a, j);
        add_g<LA, T>(lam, lqj, wjA, sg);
        if constexpr (LB > 0) add_g<LB, T>(lam + S::SA, lqj + S::SA, wjB, sg);
    }
    const T inv = T(1) / nfk;
    if constexpr (DSIG) {
        T qk[S::SQ];
        load_rec32(d.q + (size_t)k * S::SQ, qk);
        T tA = T(0), tB = T(0), uA = T(0), uB = T(0);
#pragma unroll
        for (int s = 0; s < S::SA; ++s) { tA += lam[s] * qk[s]; uA += Gk[s] * lqk[s]; }
#pragma unroll
        for (int s = S::SA; s < S::SA + S::SB; ++s) { tB += lam[s] * qk[s]; uB += Gk[s] * lqk[s]; }
        d.tu[4 * k] = tA * inv;
        d.tu[4 * k + 1] = uA;
        d.tu[4 * k + 2] = tB * inv;
        d.tu[4 * k + 3] = uB;
        store_rec(d.g + (size_t)k * S::SQ, Gk);
    }
#pragma unroll
    for (int s = 0; s < S::SQ; ++s) lam[s] *= inv;
    store_rec(d.lam + (size_t)k * S::SQ, lam);
}

// Pass 4: gather forces, f_dst = f_src - dV/dx, plus the virial block partials.
// One thread per sorted slot, or (d.iperm set) per caller index of d.i0 ..
// d.i1 - 1, so a caller-order range of f is complete when its launch is.
template <int LA, int LB, typename T, bool STEP, bool CALLER = false>
__device__ __forceinline__ void local_force_body(const LocalDev<T> &d, const double *__restrict__ f_src,
                                                 double *__restrict__ f_dst, const SysDev &s, const CellGrid &g,
                                                 double *vpart, DevStatus *status, int bid) {
    using S = LSet<LA, LB, T>;
    constexpr bool DSIG = !STEP;
    __shared__ double smem[6 * 32];
    // caller order: the block's stretch of f (3 x blockDim doubles, which
    // may be host memory over the host link) is read into shared memory and
    // written back from it with consecutive threads on consecutive doubles,
    // so every warp access is whole 128-byte lines
    __shared__ double fstage[CALLER ? 3 * kBlock : 1];
    int k, ic = 0, ib0 = 0, cnt = 0;
    bool valid;
    if constexpr (CALLER) {
        ib0 = d.i0 + bid * blockDim.x;
        cnt = max(0, min((int)blockDim.x, d.i1 - ib0));
        for (int e = threadIdx.x; e < 3 * cnt; e += blockDim.x) fstage[e] = f_src[3 * (size_t)ib0 + e];
        __syncthreads();
        ic = ib0 + threadIdx.x;
        valid = (int)threadIdx.x < cnt;
        k = valid ? d.iperm[ic] : 0;
        valid = valid && (unsigned)k < (unsigned)d.n;
    } else {
        k = bid * blockDim.x + threadIdx.x;
        valid = k < d.n;
    }
    double vir[6] = {0, 0, 0, 0, 0, 0};
    if (valid) {
        T la[S::SQ];
        load_rec(d.lam + (size_t)k * S::SQ, la);
        T qa[S::SQ], ga[S::SQ];
        T tua[4] = {T(0), T(0), T(0), T(0)};
        if constexpr (DSIG) {
            load_rec(d.q + (size_t)k * S::SQ, qa);
            load_rec(d.g + (size_t)k * S::SQ, ga);
#pragma unroll
            for (int t = 0; t < 4; ++t) tua[t] = d.tu[4 * k + t];
        }
        const auto a = d.geo.load(k);
        T gx = T(0), gy = T(0), gz = T(0);
        const int c = min(d.nb.count[k], d.nb.M);
        constexpr T sgnA = (LA & 1) ? T(-1) : T(1);
        constexpr T sgnB = (LB & 1) ? T(-1) : T(1);
        // each neighbour's index is loaded an iteration ahead, so its record
        // load waits on one memory latency instead of two
        int jn = c > 0 ? nb_index(d.nb, d.npad, 0, k) : 0;
        for (int t = 0; t < c; ++t) {
            const int j = jn;
            if (t + 1 < c) jn = nb_index(d.nb, d.npad, t + 1, k);
            T ux, uy, uz, rinv, sg, dsg;
            pair_geom<T, STEP>(d, a, j, ux, uy, uz, rinv, sg, dsg);
            T lj[S::SQ];
            load_rec32(d.lam + (size_t)j * S::SQ, lj);
            T Lm[S::SQ];
#pragma unroll
            for (int q = 0; q < S::SA; ++q) Lm[q] = la[q] + sgnA * lj[q];
#pragma unroll
            for (int q = S::SA; q < S::SQ; ++q) Lm[q] = la[q] + sgnB * lj[q];
            T ax, ay, az;
            const T sA = ylm_dot_grad<LA, T>(ux, uy, uz, rinv, Lm, ax, ay, az);
            gx -= sg * ax;
            gy -= sg * ay;
            gz -= sg * az;
            T sB = T(0);
            if constexpr (LB > 0) {
                T bx, by, bz;
                sB = ylm_dot_grad<LB, T>(ux, uy, uz, rinv, Lm + S::SA, bx, by, bz);
                gx -= sg * bx;
                gy -= sg * by;
                gz -= sg * bz;
            }
            if constexpr (DSIG) {
                if (dsg != T(0)) {
                    T qj[S::SQ], gj[S::SQ];
                    load_rec(d.q + (size_t)j * S::SQ, qj);
                    load_rec(d.g + (size_t)j * S::SQ, gj);
                    T cross = sA + sB - tua[0] - tua[1] - tua[2] - tua[3] - d.tu[4 * j] - d.tu[4 * j + 1] -
                              d.tu[4 * j + 2] - d.tu[4 * j + 3];
#pragma unroll
                    for (int q = 0; q < S::SA + S::SB; ++q) cross += ga[q] * qj[q] + gj[q] * qa[q];
                    gx -= dsg * cross * ux;
                    gy -= dsg * cross * uy;
                    gz -= dsg * cross * uz;
                }
            }
        }
        const int i = CALLER ? ic : d.perm[k];
        const double fx = -(double)gx, fy = -(double)gy, fz = -(double)gz;   // delta f = -dV/dx
        if constexpr (CALLER) {
            fstage[3 * threadIdx.x] += fx;
            fstage[3 * threadIdx.x + 1] += fy;
            fstage[3 * threadIdx.x + 2] += fz;
        } else if ((unsigned)i < (unsigned)d.n) {   // a sorted order left by a rebuild that gave up is not trusted
            f_dst[3 * i] = f_src[3 * i] + fx;
            f_dst[3 * i + 1] = f_src[3 * i + 1] + fy;
            f_dst[3 * i + 2] = f_src[3 * i + 2] + fz;
        }
        if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) atomicOr(&status->nan_force, 1u);
        if (vpart && (unsigned)i < (unsigned)d.n) {
            double ux_ = s.xs[3 * k], uy_ = s.xs[3 * k + 1], uz_ = s.xs[3 * k + 2];
            if (s.image) {
                int ix, iy, iz;
                unpack_image(s.image[i], ix, iy, iz);
                ux_ += ix * g.L[0];
                uy_ += iy * g.L[1];
                uz_ += iz * g.L[2];
            }
            vir[0] = fx * ux_; vir[1] = fy * uy_; vir[2] = fz * uz_;
            vir[3] = fx * uy_; vir[4] = fx * uz_; vir[5] = fy * uz_;
        }
    }
    if constexpr (CALLER) {
        __syncthreads();
        for (int e = threadIdx.x; e < 3 * cnt; e += blockDim.x) f_dst[3 * (size_t)ib0 + e] = fstage[e];
    }
    if (vpart) {
        block_sum<6>(vir, smem);
        if (threadIdx.x == 0)
            for (int t = 0; t < 6; ++t) vpart[bid * 8 + t] = vir[t];
    }
}


}  // namespace mtd
