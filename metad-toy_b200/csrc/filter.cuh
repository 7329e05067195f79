// filter.cuh -- the exact neighbour decision shared by the per-step neighbour
// search and the skin-list filter.
//
// A candidate is decided by its FP32 cell-relative r^2 unless that lies
// within the guard band [lo2, hi2] around the bound; inside the band the FP64
// test on raw coordinates decides with the FP64 oracle's operations in the
// same order, so every neighbour set equals the FP64 criterion exactly.
#pragma once

#include "kernels.h"

namespace mtd {

// What the FP64 decision reads, taken by value by the out-of-line test: a
// reference into a kernel parameter passed to a non-inlined function makes
// every thread copy the whole parameter block to its stack at kernel entry.
struct ExactSpec {
    double L[3], invL[3];
    int periodic[3];
    double rc2, r0, eps;
    SwParams sw;
};
__device__ __forceinline__ ExactSpec exact_spec(const GeoD &gd, const NeighSpec &ns) {
    ExactSpec e;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        e.L[c] = gd.L[c];
        e.invL[c] = gd.invL[c];
        e.periodic[c] = gd.periodic[c];
    }
    e.rc2 = ns.rc2;
    e.r0 = ns.r0;
    e.eps = ns.eps;
    e.sw = ns.sw;
    return e;
}

// FP64 decision on the raw coordinates of sorted atoms k and j (the oracle's
// criterion, operation by operation).  Out of line: the guard band is rare,
// and its FP64 registers stay out of the callers' loops.
template <int KIND>
__device__ __noinline__ bool exact_decide(const ExactSpec e, const double *__restrict__ xs, int k, int j) {
    GeoD gd;
    gd.xs = xs;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        gd.L[c] = e.L[c];
        gd.invL[c] = e.invL[c];
        gd.periodic[c] = e.periodic[c];
    }
    const double xk[3] = {xs[3 * k], xs[3 * k + 1], xs[3 * k + 2]};
    const double xj[3] = {xs[3 * j], xs[3 * j + 1], xs[3 * j + 2]};
    double d[3];
    const double r2 = exact_disp(gd, xk, xj, d);
    if (KIND == NK_RANGE) return (r2 <= e.rc2) && (r2 >= 1e-12);
    if (KIND == NK_STEP) return (r2 <= e.rc2) && (__dsqrt_rn(r2) < e.r0);
    return (r2 <= e.rc2) && (sw_f<double>(e.sw, __dsqrt_rn(r2)) >= e.eps);
}

// The decision for a candidate at FP32 squared distance r2f.
template <int KIND>
__device__ __forceinline__ bool decide(const GeoD &gd, const NeighSpec &ns, const double *xs, int k, int j,
                                       float r2f) {
    if (r2f > ns.hi2) return false;
    if (KIND != NK_SWITCH && r2f < ns.lo2 && r2f > 1e-6f) return true;
    return exact_decide<KIND>(exact_spec(gd, ns), xs, k, j);
}

// Skin-list filter of sorted atom k: the candidates found within cutoff +
// skin at the last rebuild, tested against the exact criterion at the
// current positions, kept in candidate order into nd.list / nd.count.
// Returns the kept count (which may exceed nd.M: overflow, reported).
template <int KIND>
__device__ __forceinline__ int filter_atom(const GeoF &gf, const GeoD &gd, const double *xs, const NeighSpec &ns,
                                           const NeighDev &cand, const NeighDev &nd, int npad, int k,
                                           DevStatus *status) {
    const float4 a = __ldg(gf.pf + k);
    const int nc = min(__ldg(cand.count + k), cand.M);
    int cnt = 0;
    int jn = nc > 0 ? __ldg(cand.list + k) : 0;
    float4 bn = nc > 0 ? __ldg(gf.pf + jn) : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int t = 0; t < nc; ++t) {
        const int j = jn;
        const float4 b = bn;
        if (t + 1 < nc) {   // the next candidate's index and position in flight
            jn = __ldg(cand.list + (size_t)(t + 1) * npad + k);
            bn = __ldg(gf.pf + jn);
        }
        float dx, dy, dz;
        disp_f(gf, a, b, dx, dy, dz);
        const float r2f = dx * dx + dy * dy + dz * dz;
        if (!decide<KIND>(gd, ns, xs, k, j, r2f)) continue;
        if (cnt < nd.M) nd.list[(size_t)cnt * npad + k] = j;
        ++cnt;
    }
    nd.count[k] = cnt;
    if (cnt > nd.M) atomicMax(&status->overflow, (unsigned)cnt);
    return cnt;
}

}  // namespace mtd
