// geo.cuh -- pair displacements from the sorted per-atom positions.
//
// Mixed precision keeps every atom as an FP32 offset from the lower corner of
// its cell plus the packed cell coordinates (10 bits each).  A displacement is
//   d = dcell * h + (off_j - off_i),  dcell wrapped to the nearest image,
// so its error is a few ulp of the cell size (~1e-7 relative at 3.9 A cells)
// rather than of the box length.  FP64 mode uses the caller's raw coordinates
// with the FP64 minimum image the neighbour decision uses.
#pragma once

#include "common.cuh"

namespace mtd {

__device__ __forceinline__ int pack_cell(int cx, int cy, int cz) { return cx | (cy << 10) | (cz << 20); }

struct GeoF {
    const float4 *pf;
    float hf[3], Lf[3], invLf[3];
    int nc[3], periodic[3];
};

struct GeoD {
    const double *xs;
    double L[3], invL[3];
    int periodic[3];
};

// Minimum-image displacement x_j - x_i in FP64 without FMA contraction; the
// FP64 oracle performs the same operations in the same order.
__device__ __forceinline__ double exact_disp(const GeoD &g, const double *xi, const double *xj, double *d) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double t = __dsub_rn(xj[c], xi[c]);
        if (g.periodic[c]) {
            const double k = rint(__dmul_rn(t, g.invL[c]));
            t = __dsub_rn(t, __dmul_rn(g.L[c], k));
        }
        d[c] = t;
    }
    return __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2]));
}

__device__ __forceinline__ void disp_f(const GeoF &g, const float4 &a, const float4 &b, float &dx, float &dy,
                                       float &dz) {
    const int wa = __float_as_int(a.w), wb = __float_as_int(b.w);
    int dc[3] = {(wb & 1023) - (wa & 1023), ((wb >> 10) & 1023) - ((wa >> 10) & 1023), (wb >> 20) - (wa >> 20)};
    const float off[3] = {b.x - a.x, b.y - a.y, b.z - a.z};
    float d[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        int e = dc[c];
        if (g.periodic[c]) {
            if (e > 1) e -= g.nc[c];
            else if (e < -1) e += g.nc[c];
        }
        float t = (float)e * g.hf[c] + off[c];
        if (g.periodic[c]) t -= g.Lf[c] * rintf(t * g.invLf[c]);
        d[c] = t;
    }
    dx = d[0];
    dy = d[1];
    dz = d[2];
}

// Precision-generic view used by the CV kernels.
template <typename T> struct Geo;

template <> struct Geo<float> {
    GeoF g;
    using Pos = float4;
    __device__ __forceinline__ Pos load(int i) const { return __ldg(g.pf + i); }
    __device__ __forceinline__ void disp(const Pos &a, const Pos &b, float &dx, float &dy, float &dz) const {
        disp_f(g, a, b, dx, dy, dz);
    }
};

template <> struct Geo<double> {
    GeoD g;
    struct Pos {
        double v[3];
    };
    __device__ __forceinline__ Pos load(int i) const {
        Pos p;
        p.v[0] = g.xs[3 * i];
        p.v[1] = g.xs[3 * i + 1];
        p.v[2] = g.xs[3 * i + 2];
        return p;
    }
    __device__ __forceinline__ void disp(const Pos &a, const Pos &b, double &dx, double &dy, double &dz) const {
        double d[3];
        exact_disp(g, a.v, b.v, d);
        dx = d[0];
        dy = d[1];
        dz = d[2];
    }
};

}  // namespace mtd
