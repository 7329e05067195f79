// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference project's own spherical-harmonic arithmetic
// (include/CVsets/CV_Steinhardt_math.h of Metad-toy) as host C++ and exposes it
// through a C ABI, so that the oracle's restatement can be pinned against the
// reference code itself.  The header is read from the reference checkout at
// build time (oracle/Makefile, target `ref`); nothing of it is copied here.
//
// Angle preparation follows the kernels that call these functions:
//   theta = acos(dz/r), phi = atan2(dy, dx), sincos(k*theta), sincos(k*phi)
//   (src/cvs/CVs_Steinhardt.cu:1441-1475, :1571-1600).
#include <cmath>

// The reference header is CUDA device code; compile it for the host.
#define __device__
#define __forceinline__ inline
// Power helpers with the meaning of include/utils/zqc_debug.h:3-8.
#define POW2(a) ((a) * (a))
#define POW3(a) ((a) * (a) * (a))
#define POW4(a) ((a) * (a) * (a) * (a))
#define POW5(a) ((a) * (a) * (a) * (a) * (a))
#define POW6(a) (POW3(a) * POW3(a))
#define POW7(a) (POW3(a) * POW4(a))

#include "CV_Steinhardt_math.h"

namespace {
struct Angles {
    double r;
    double ct[8], st[8], cp[8], sp[8];  // cos/sin of k*theta and k*phi, k = 0..7
};

Angles angles(double dx, double dy, double dz) {
    Angles a;
    a.r = std::sqrt(dx * dx + dy * dy + dz * dz);
    double theta = std::acos(std::fmax(-1.0, std::fmin(1.0, dz / a.r)));
    double phi = std::atan2(dy, dx);
    for (int k = 0; k < 8; k++) {
        a.st[k] = std::sin(k * theta);
        a.ct[k] = std::cos(k * theta);
        a.sp[k] = std::sin(k * phi);
        a.cp[k] = std::cos(k * phi);
    }
    return a;
}
}  // namespace

extern "C" {

// Y_lm, m = 0..l as (re, im) pairs: compute_Ylm_forward_L{3,4,6}.
int ref_ylm(int l, double dx, double dy, double dz, double *out) {
    Angles a = angles(dx, dy, dz);
    if (l == 3) {
        compute_Ylm_forward_L3(a.ct[1], a.st[1], a.cp[1], a.sp[1], a.ct[2], a.st[2], a.cp[2], a.sp[2],
                               a.ct[3], a.st[3], a.cp[3], a.sp[3], out);
    } else if (l == 4) {
        compute_Ylm_forward_L4(a.ct[1], a.st[1], a.cp[1], a.sp[1], a.cp[2], a.sp[2], a.cp[3], a.sp[3],
                               a.cp[4], a.sp[4], out);
    } else if (l == 6) {
        compute_Ylm_forward_L6(a.ct[1], a.st[1], a.cp[1], a.sp[1], a.ct[2], a.st[2], a.cp[2], a.sp[2],
                               a.cp[3], a.sp[3], a.ct[4], a.st[4], a.cp[4], a.sp[4], a.cp[5], a.sp[5],
                               a.ct[6], a.st[6], a.cp[6], a.sp[6], out);
    } else {
        return 1;
    }
    return 0;
}

// dY_lm / d(displacement): compute_dYlmdx_gradient_L{4,6}; out[6*m + {dx_re, dx_im, dy_re, dy_im, dz_re, dz_im}].
int ref_dylm(int l, double dx, double dy, double dz, double *out) {
    Angles a = angles(dx, dy, dz);
    if (l == 4) {
        MetaD_zqc::D_Ylm_Layout<4> lay;
        compute_dYlmdx_gradient_L4(a.r, a.ct[1], a.st[1], a.cp[1], a.sp[1], a.ct[2], a.st[2], a.cp[2], a.sp[2],
                                   a.ct[3], a.st[3], a.cp[3], a.sp[3], a.ct[4], a.st[4], a.cp[4], a.sp[4],
                                   a.ct[5], a.st[5], a.cp[5], a.sp[5], a.ct[6], a.st[6], &lay);
        const MetaD_zqc::Ylm_Entry *e = &lay.Y40;
        for (int m = 0; m <= 4; m++) {
            out[6 * m + 0] = e[m].dx_re; out[6 * m + 1] = e[m].dx_im;
            out[6 * m + 2] = e[m].dy_re; out[6 * m + 3] = e[m].dy_im;
            out[6 * m + 4] = e[m].dz_re; out[6 * m + 5] = e[m].dz_im;
        }
    } else if (l == 6) {
        MetaD_zqc::D_Ylm_Layout<6> lay;
        compute_dYlmdx_gradient_L6(a.r, a.ct[1], a.st[1], a.cp[1], a.sp[1], a.ct[2], a.st[2], a.cp[2], a.sp[2],
                                   a.ct[3], a.st[3], a.cp[3], a.sp[3], a.ct[4], a.st[4], a.cp[4], a.sp[4],
                                   a.ct[5], a.st[5], a.cp[5], a.sp[5], a.ct[6], a.st[6], a.cp[6], a.sp[6], &lay);
        const MetaD_zqc::Ylm_Entry *e = &lay.Y60;
        for (int m = 0; m <= 6; m++) {
            out[6 * m + 0] = e[m].dx_re; out[6 * m + 1] = e[m].dx_im;
            out[6 * m + 2] = e[m].dy_re; out[6 * m + 3] = e[m].dy_im;
            out[6 * m + 4] = e[m].dz_re; out[6 * m + 5] = e[m].dz_im;
        }
    } else {
        return 1;
    }
    return 0;
}

// Reference STEINH Q AVE gradient, restating the loop of steinhardt_dcv_AVE_kernel
// (src/cvs/CVs_Steinhardt.cu:1538-1692) around the reference's own per-pair
// compute_Ylm_gradient_L{4,6}.  Inputs are the kept neighbour lists (n*cap, -1 padded),
// their counts, q_lm (n * 2(l+1)), Q (n) and the group mask; group = all atoms is assumed
// exactly as the reference kernel assumes it (index mixing noted at :1561-1562).
// `disp` holds the per-pair displacement (n*cap*3).  Output dcvdx (n*3).
int ref_q_grad_faithful(int l, int n, int cap, const int *kept, const int *nkept, const double *disp,
                        const double *qlm_in, const double *Q, const int *ingroup, int all_count,
                        double *dcvdx) {
    if (l != 4 && l != 6) return 1;
    const int S = 2 * (l + 1);
    double *qlm = const_cast<double *>(qlm_in);
    for (int i = 0; i < n; i++) {
        double acc[6] = {0, 0, 0, 0, 0, 0};
        dcvdx[3 * i] = dcvdx[3 * i + 1] = dcvdx[3 * i + 2] = 0.0;
        int nn = nkept[i];
        if (nn == 0) continue;
        double catom = 1.0 / (Q[i] * nn);
        for (int t = 0; t < nn; t++) {
            const double *d = disp + ((long)i * cap + t) * 3;
            Angles a = angles(d[0], d[1], d[2]);
            int j = kept[(long)i * cap + t];
            double neigh = 0.0;
            int jbase = 0;
            if (ingroup[j]) {
                neigh = 1.0 / (Q[j] * nkept[j]);
                jbase = j * S;
            }
            if (l == 4) {
                compute_Ylm_gradient_L4(a.r, a.ct[1], a.st[1], a.cp[1], a.sp[1], a.ct[2], a.st[2], a.cp[2], a.sp[2],
                                        a.ct[3], a.st[3], a.cp[3], a.sp[3], a.ct[4], a.st[4], a.cp[4], a.sp[4],
                                        a.ct[5], a.st[5], a.cp[5], a.sp[5], a.ct[6], a.st[6], catom, neigh,
                                        i * S, jbase, qlm, acc);
            } else {
                compute_Ylm_gradient_L6(a.r, a.ct[1], a.st[1], a.cp[1], a.sp[1], a.ct[2], a.st[2], a.cp[2], a.sp[2],
                                        a.ct[3], a.st[3], a.cp[3], a.sp[3], a.ct[4], a.st[4], a.cp[4], a.sp[4],
                                        a.ct[5], a.st[5], a.cp[5], a.sp[5], a.ct[6], a.st[6], a.cp[6], a.sp[6],
                                        catom, neigh, i * S, jbase, qlm, acc);
            }
        }
        const double pi = 3.1415926535897932385;
        for (int c = 0; c < 3; c++) {
            double v = acc[2 * c] + acc[2 * c + 1];
            dcvdx[3 * i + c] = -(v * 2 * pi) / (all_count * (2 * l + 1));
        }
    }
    return 0;
}

}  // extern "C"
