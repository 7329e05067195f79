// ylm.cuh -- spherical harmonics Y_lm (m = 0..l) from the unit bond vector
// without trigonometric functions:
//
//   Y_lm(u) = C_lm * D_lm(u_z) * (u_x + i u_y)^m,
//   D_lm = d^m P_l / dz^m,   C_lm = (-1)^m sqrt((2l+1)/(4 pi) (l-m)!/(l+m)!).
//
// This is the orthonormal, Condon-Shortley-phased basis of the reference's
// closed forms (include/CVsets/CV_Steinhardt_math.h:981-1217); the q_lm layout
// [Re m=0, Im m=0, Re m=1, Im m=1, ...] matches the reference's 2(l+1) storage.
// The gradient with respect to the displacement d (|d| = r) is obtained from
// the polynomial extension Yhat(u) as  (1/r) (I - u u^T) grad_u Yhat, with
//   dYhat/du_x = C D m w^(m-1),  dYhat/du_y = i C D m w^(m-1),
//   dYhat/du_z = C D_{l,m+1} w^m.
// Coefficients are compile-time constants (constexpr, unrolled by templates).
#pragma once

#include "common.cuh"

#include <type_traits>
#include <utility>

namespace mtd {
namespace ylm_detail {

constexpr double cfact(int n) {
    double r = 1.0;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
}
constexpr double cpow2(int n) {
    double r = 1.0;
    for (int i = 0; i < n; ++i) r *= 2.0;
    return r;
}
constexpr double csqrt(double x) {
    if (x <= 0.0) return 0.0;
    double g = x > 1.0 ? x : 1.0;
    for (int i = 0; i < 200; ++i) g = 0.5 * (g + x / g);
    return g;
}
// Coefficient of z^k in the Legendre polynomial P_l.
constexpr double leg(int l, int k) {
    if (k < 0 || k > l || ((l - k) & 1)) return 0.0;
    const int j = (l - k) / 2;
    const double s = (j & 1) ? -1.0 : 1.0;
    return s * cfact(2 * l - 2 * j) / (cpow2(l) * cfact(j) * cfact(l - j) * cfact(l - 2 * j));
}
// Coefficient of z^k in D_lm = d^m P_l / dz^m.
constexpr double dcoef(int l, int m, int k) { return leg(l, k + m) * cfact(k + m) / cfact(k); }
constexpr double cnorm(int l, int m) {
    return ((m & 1) ? -1.0 : 1.0) * csqrt((2.0 * l + 1.0) / (4.0 * kPi) * cfact(l - m) / cfact(l + m));
}

// Horner step over z^2 with the normalisation C_lm folded into the coefficient.
template <int L, int M, int K, typename T> struct Horner {
    __device__ __host__ static __forceinline__ T run(T z2, T acc) {
        constexpr double c = dcoef(L, M, K) * cnorm(L, M);
        acc = acc * z2 + T(c);
        if constexpr (K >= 2) return Horner<L, M, K - 2, T>::run(z2, acc);
        else return acc;
    }
};

template <int I, int N, typename F> __device__ __host__ __forceinline__ void static_for(F &&f) {
    if constexpr (I < N) {
        f(std::integral_constant<int, I>{});
        static_for<I + 1, N>(f);
    }
}

}  // namespace ylm_detail

// D_lm(z) including C_lm; zero for M > L.
template <int L, int M, typename T> __device__ __host__ __forceinline__ T cdpoly(T z, T z2) {
    using namespace ylm_detail;
    if constexpr (M > L) {
        return T(0);
    } else {
        constexpr int deg = L - M;
        constexpr double top = dcoef(L, M, deg) * cnorm(L, M);
        T acc = T(top);
        if constexpr (deg >= 2) acc = Horner<L, M, deg - 2, T>::run(z2, acc);
        if constexpr (deg & 1) acc *= z;
        return acc;
    }
}

// Y_lm for m = 0..L, accumulated with weight wgt: acc[2m] += wgt Re Y, acc[2m+1] += wgt Im Y.
template <int L, typename T>
__device__ __host__ __forceinline__ void ylm_accum(T ux, T uy, T uz, T wgt, T *acc) {
    using namespace ylm_detail;
    const T z2 = uz * uz;
    T wr = T(1), wi = T(0);
    static_for<0, L + 1>([&](auto mc) {
        constexpr int m = decltype(mc)::value;
        const T c = wgt * cdpoly<L, m, T>(uz, z2);
        acc[2 * m] += c * wr;
        if constexpr (m > 0) acc[2 * m + 1] += c * wi;
        const T nr = wr * ux - wi * uy;
        const T ni = wr * uy + wi * ux;
        wr = nr;
        wi = ni;
    });
}

// Value s = sum_m (Lam_re Re Y + Lam_im Im Y) and the gradient of s with respect
// to the displacement d (u = d/r, rinv = 1/r).
template <int L, typename T>
__device__ __host__ __forceinline__ T ylm_dot_grad(T ux, T uy, T uz, T rinv, const T *lam, T &gx, T &gy, T &gz) {
    using namespace ylm_detail;
    const T z2 = uz * uz;
    T wr = T(1), wi = T(0);   // w^m
    T pr = T(0), pi = T(0);   // w^(m-1)
    T s = T(0), hx = T(0), hy = T(0), hz = T(0);
    T Dm = cdpoly<L, 0, T>(uz, z2);
    static_for<0, L + 1>([&](auto mc) {
        constexpr int m = decltype(mc)::value;
        // D_{l,m+1} carries C_{l,m+1}; rescale to C_{l,m} for the u_z derivative.
        constexpr double ratio = (m + 1 <= L) ? cnorm(L, m) / cnorm(L, m + 1) : 0.0;
        const T Dm1 = cdpoly<L, m + 1, T>(uz, z2);
        const T lr = lam[2 * m];
        const T li = (m > 0) ? lam[2 * m + 1] : T(0);
        const T a = lr * wr + li * wi;               // Re(conj-free contraction with w^m)
        s += Dm * a;
        hz += T(ratio) * Dm1 * a;
        if constexpr (m > 0) {
            const T b = T(m) * Dm;
            hx += b * (lr * pr + li * pi);
            hy += b * (li * pr - lr * pi);
        }
        pr = wr;
        pi = wi;
        const T nr = wr * ux - wi * uy;
        const T ni = wr * uy + wi * ux;
        wr = nr;
        wi = ni;
        Dm = Dm1;
    });
    const T uh = ux * hx + uy * hy + uz * hz;
    gx = (hx - ux * uh) * rinv;
    gy = (hy - uy * uh) * rinv;
    gz = (hz - uz * uh) * rinv;
    return s;
}

}  // namespace mtd
