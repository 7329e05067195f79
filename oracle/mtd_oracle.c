/*
 * mtd_oracle.c -- CPU FP64 restatement of the Metad-toy metadynamics hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see mtd_oracle.h).  Compiled with
 * -ffp-contract=off so that the displacement and r^2 arithmetic rounds
 * exactly like the product's FP64 neighbour test.
 *
 * Citations are file:line in the Metad-toy reference project.
 */
#include "mtd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846
#define ORC_LMAX 12

static int g_threads = 0;
void orc_set_threads(int nthreads) { g_threads = nthreads; }
int orc_get_threads(void) {
#ifdef _OPENMP
    return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_free(void *p) { free(p); }

/* ------------------------------------------------------------------------- */
/* Switching functions: include/utils/zqc_switch_function.h:163-313, :339-367 */
/* ------------------------------------------------------------------------- */
static double ipow(double x, int n) { return pow(x, (double)n); }

double orc_sw_f(const orc_sw *p, double x) {
    switch (p->type) {
    case 0: return 1.0;                                   /* LINE  :168-171 */
    case 1: return (x < p->r0) ? 1.0 : 0.0;              /* STEP  :220-226 */
    case 2: return 1.0 / (1.0 + exp(-p->alpha * (x - p->r0)));       /* FERMI */
    case 3: return 0.5 * (1.0 + tanh(p->alpha * (x - p->r0)));       /* TANH  */
    case 4: {                                                          /* RATIONAL :251-271 */
        int n = p->n, m = p->m;
        double y = (x - p->d0) / p->r0;
        if (n == 6 && m == 12) { double y2 = y * y; double y6 = y2 * y2 * y2; return 1.0 / (1.0 + y6); }
        if (n == 4 && m == 8) { double y2 = y * y; double y4 = y2 * y2; return 1.0 / (1.0 + y4); }
        if (2 * n == m) return 1.0 / (1.0 + ipow(y, n));
        if (n == 2 * m) return 1.0 + ipow(y, m);   /* reference returns (1 + x^m) here, kept as is */
        return (1.0 - ipow(y, n)) / (1.0 - ipow(y, m));
    }
    default: return 1.0;
    }
}

double orc_sw_df(const orc_sw *p, double x) {
    switch (p->type) {
    case 0: return 0.0;
    case 1: return 0.0;
    case 2: { double e = exp(-p->alpha * (x - p->r0)); double den = 1.0 + e; return (p->alpha * e) / (den * den); }
    case 3: { double t = tanh(p->alpha * (x - p->r0)); return 0.5 * p->alpha * (1.0 - t * t); }
    case 4: {                                                          /* :273-313 */
        int n = p->n, m = p->m;
        double y = (x - p->d0) / p->r0;
        if (n == 6 && m == 12) {
            double y2 = y * y, y5 = y2 * y2 * y, y6 = y2 * y2 * y2;
            return -n * y5 / ((1.0 + y6) * (1.0 + y6)) / p->r0;
        }
        if (n == 4 && m == 8) {
            double y2 = y * y, y3 = y2 * y, y4 = y2 * y2;
            return -(double)n * y3 / ((1.0 + y4) * (1.0 + y4)) / p->r0;
        }
        if (2 * n == m) {
            double a = ipow(y, n - 1), b = ipow(y, n);
            return -(double)n * a / ((1.0 + b) * (1.0 + b)) / p->r0;
        }
        if (n == 2 * m) return (double)m * ipow(y, m - 1) / p->r0;
        {
            double ymm1 = ipow(y, m - 1), ym = ymm1 * y;
            if (fabs(1.0 - ym) < 1e-12) return -0.5 * (double)(n * (n - m)) / (double)m / p->r0;
            double ynm1 = ipow(y, n - 1);
            return ((double)(n - m) * ynm1 * ym + m * ymm1 - n * ynm1) / ((1 - ym) * (1 - ym)) / p->r0;
        }
    }
    default: return 0.0;
    }
}

double orc_sw_invert_for_eps(const orc_sw *p, double eps) {   /* :339-367 */
    switch (p->type) {
    case 1: return p->r0;
    case 2: return p->r0 - log(1.0 / eps - 1.0) / p->alpha;
    case 3: return p->r0 + atanh(2.0 * eps - 1.0) / p->alpha;
    case 4:
        if (p->n == 6 && p->m == 12) return pow(1.0 / eps - 1.0, 1.0 / 6.0) * p->r0 + p->d0;
        if (p->n == 4 && p->m == 8) return pow(1.0 / eps - 1.0, 1.0 / 4.0) * p->r0 + p->d0;
        if (2 * p->n == p->m) return pow(1.0 / eps - 1.0, 1.0 / p->n) * p->r0 + p->d0;
        {   /* bisection, :318-337 */
            double lo = 0.0, hi = 1.0;
            while (orc_sw_f(p, hi) > eps) { hi *= 2.0; if (hi > 1e8) break; }
            for (int it = 0; it < 100; it++) {
                double mid = 0.5 * (lo + hi);
                if (orc_sw_f(p, mid) > eps) lo = mid; else hi = mid;
            }
            return 0.5 * (lo + hi);
        }
    default: return -1.0;
    }
}

/* ------------------------------------------------------------------------- */
/* Spherical harmonics by the associated-Legendre definition                  */
/*   Y_lm(u) = (-1)^m N_lm (d^m P_l / dz^m)(u_z) (u_x + i u_y)^m              */
/* ------------------------------------------------------------------------- */
static double g_dpoly[ORC_LMAX + 1][ORC_LMAX + 2][ORC_LMAX + 1];
static double g_cnorm[ORC_LMAX + 1][ORC_LMAX + 1];
static int g_tables_ready = 0;

static void init_tables(void) {
    if (g_tables_ready) return;
    double P[ORC_LMAX + 1][ORC_LMAX + 1];
    memset(P, 0, sizeof(P));
    P[0][0] = 1.0;
    P[1][1] = 1.0;
    for (int n = 1; n < ORC_LMAX; n++)   /* (n+1) P_{n+1} = (2n+1) z P_n - n P_{n-1} */
        for (int k = 0; k <= ORC_LMAX; k++) {
            double v = -(double)n * P[n - 1][k];
            if (k > 0) v += (2.0 * n + 1.0) * P[n][k - 1];
            P[n + 1][k] = v / (n + 1.0);
        }
    memset(g_dpoly, 0, sizeof(g_dpoly));
    for (int l = 0; l <= ORC_LMAX; l++) {
        for (int k = 0; k <= ORC_LMAX; k++) g_dpoly[l][0][k] = P[l][k];
        for (int m = 1; m <= l + 1; m++)
            for (int k = 0; k < ORC_LMAX; k++) g_dpoly[l][m][k] = (k + 1) * g_dpoly[l][m - 1][k + 1];
        for (int m = 0; m <= l; m++) {
            double ratio = 1.0;   /* (l-m)!/(l+m)! */
            for (int t = l - m + 1; t <= l + m; t++) ratio /= t;
            double nlm = sqrt((2.0 * l + 1.0) / (4.0 * ORC_PI) * ratio);
            g_cnorm[l][m] = (m % 2 ? -1.0 : 1.0) * nlm;
        }
    }
    g_tables_ready = 1;
}

static double dpoly_eval(int l, int m, double z) {
    if (m > l) return 0.0;
    double acc = 0.0;
    for (int k = l - m; k >= 0; k--) acc = acc * z + g_dpoly[l][m][k];
    return acc;
}

void orc_ylm(int l, const double d[3], double *yre, double *yim) {
    init_tables();
    double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double ux = d[0] / r, uy = d[1] / r, uz = d[2] / r;
    double wr = 1.0, wi = 0.0;
    for (int m = 0; m <= l; m++) {
        double c = g_cnorm[l][m] * dpoly_eval(l, m, uz);
        yre[m] = c * wr;
        yim[m] = c * wi;
        double nr = wr * ux - wi * uy, ni = wr * uy + wi * ux;
        wr = nr; wi = ni;
    }
}

void orc_ylm_grad(int l, const double d[3], double *yre, double *yim, double *gre, double *gim) {
    init_tables();
    double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double u[3] = {d[0] / r, d[1] / r, d[2] / r};
    double wr = 1.0, wi = 0.0;       /* w^m */
    double pr = 0.0, pi = 0.0;       /* w^(m-1) */
    for (int m = 0; m <= l; m++) {
        double Dm = dpoly_eval(l, m, u[2]);
        double Dm1 = dpoly_eval(l, m + 1, u[2]);
        double C = g_cnorm[l][m];
        yre[m] = C * Dm * wr;
        yim[m] = C * Dm * wi;
        /* gradient of the polynomial extension in u */
        double hr[3], hi[3];
        hr[0] = C * Dm * m * pr;   hi[0] = C * Dm * m * pi;
        hr[1] = -C * Dm * m * pi;  hi[1] = C * Dm * m * pr;      /* i * w^(m-1) */
        hr[2] = C * Dm1 * wr;      hi[2] = C * Dm1 * wi;
        double ur = u[0] * hr[0] + u[1] * hr[1] + u[2] * hr[2];
        double ui = u[0] * hi[0] + u[1] * hi[1] + u[2] * hi[2];
        for (int c = 0; c < 3; c++) {
            gre[m * 3 + c] = (hr[c] - u[c] * ur) / r;
            gim[m * 3 + c] = (hi[c] - u[c] * ui) / r;
        }
        pr = wr; pi = wi;
        double nr = wr * u[0] - wi * u[1], ni = wr * u[1] + wi * u[0];
        wr = nr; wi = ni;
    }
}

/* ------------------------------------------------------------------------- */
/* Geometry                                                                   */
/* ------------------------------------------------------------------------- */
void orc_minimg(const orc_box *b, const double *xi, const double *xj, double *d) {
    for (int c = 0; c < 3; c++) {
        double t = xj[c] - xi[c];
        if (b->periodic[c]) {
            double inv = 1.0 / b->L[c];
            double k = rint(t * inv);
            double s = b->L[c] * k;
            t = t - s;
        }
        d[c] = t;
    }
}

double orc_r2(const double *d) {
    double a = d[0] * d[0];
    double b = d[1] * d[1];
    double c = d[2] * d[2];
    double s = a + b;
    return s + c;
}

typedef struct { int nc[3]; double lo[3], h[3]; int *head, *next; } cellgrid;

static void cells_build(cellgrid *g, int n, const double *x, const orc_box *box, double rcut) {
    for (int c = 0; c < 3; c++) {
        double lo, ext;
        if (box->periodic[c]) { lo = 0.0; ext = box->L[c]; }
        else {
            lo = 1e300; double hi = -1e300;
            for (int i = 0; i < n; i++) { if (x[3 * i + c] < lo) lo = x[3 * i + c]; if (x[3 * i + c] > hi) hi = x[3 * i + c]; }
            if (n == 0) { lo = 0; hi = 0; }
            ext = hi - lo;
        }
        int nc = (rcut > 0) ? (int)floor(ext / rcut) : 1;
        if (nc < 1) nc = 1;
        if (nc > 1024) nc = 1024;
        g->nc[c] = nc; g->lo[c] = lo; g->h[c] = (ext > 0 ? ext / nc : 1.0);
    }
    int ncell = g->nc[0] * g->nc[1] * g->nc[2];
    g->head = (int *)malloc(sizeof(int) * ncell);
    g->next = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    for (int i = 0; i < ncell; i++) g->head[i] = -1;
    for (int i = n - 1; i >= 0; i--) {
        int ci[3];
        for (int c = 0; c < 3; c++) {
            double v = x[3 * i + c] - g->lo[c];
            if (box->periodic[c]) { v = v - box->L[c] * floor(v / box->L[c]); }
            int k = (int)floor(v / g->h[c]);
            if (k < 0) k = 0;
            if (k >= g->nc[c]) k = g->nc[c] - 1;
            ci[c] = k;
        }
        int cell = (ci[0] * g->nc[1] + ci[1]) * g->nc[2] + ci[2];
        g->next[i] = g->head[cell];
        g->head[cell] = i;
    }
}

static int cell_of(const cellgrid *g, const orc_box *box, const double *xi, int *ci) {
    for (int c = 0; c < 3; c++) {
        double v = xi[c] - g->lo[c];
        if (box->periodic[c]) v = v - box->L[c] * floor(v / box->L[c]);
        int k = (int)floor(v / g->h[c]);
        if (k < 0) k = 0;
        if (k >= g->nc[c]) k = g->nc[c] - 1;
        ci[c] = k;
    }
    return 0;
}

static int stencil(const cellgrid *g, const orc_box *box, int c, int ci, int *out) {
    int nc = g->nc[c], cnt = 0;
    if (nc == 1) { out[0] = 0; return 1; }
    if (box->periodic[c]) {
        if (nc == 2) { out[0] = 0; out[1] = 1; return 2; }
        for (int o = -1; o <= 1; o++) out[cnt++] = ((ci + o) % nc + nc) % nc;
        return cnt;
    }
    for (int o = -1; o <= 1; o++) if (ci + o >= 0 && ci + o < nc) out[cnt++] = ci + o;
    return cnt;
}

static int cmp_int(const void *a, const void *b) { int x = *(const int *)a, y = *(const int *)b; return (x > y) - (x < y); }

static int pairs_row(const cellgrid *g, const orc_box *box, const double *x, int i, double rc2, int *buf, int cap) {
    int ci[3], sx[3], sy[3], sz[3];
    cell_of(g, box, x + 3 * i, ci);
    int nx = stencil(g, box, 0, ci[0], sx), ny = stencil(g, box, 1, ci[1], sy), nz = stencil(g, box, 2, ci[2], sz);
    int cnt = 0;
    for (int a = 0; a < nx; a++) for (int b = 0; b < ny; b++) for (int c = 0; c < nz; c++) {
        int cell = (sx[a] * g->nc[1] + sy[b]) * g->nc[2] + sz[c];
        for (int j = g->head[cell]; j >= 0; j = g->next[j]) {
            if (j == i) continue;
            double d[3];
            orc_minimg(box, x + 3 * i, x + 3 * j, d);
            if (orc_r2(d) <= rc2) { if (cnt < cap) buf[cnt] = j; cnt++; }
        }
    }
    if (cnt <= cap) qsort(buf, cnt, sizeof(int), cmp_int);
    return cnt;
}

int orc_pairs(int n, const double *x, const orc_box *box, double rcut, int64_t **off_out, int **nbr_out) {
    cellgrid g;
    cells_build(&g, n, x, box, rcut);
    double rc2 = rcut * rcut;
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    int *cnt = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int nth = orc_get_threads();
#pragma omp parallel num_threads(nth)
    {
        int cap = 4096;
        int *buf = (int *)malloc(sizeof(int) * cap);
#pragma omp for schedule(static)
        for (int i = 0; i < n; i++) cnt[i] = pairs_row(&g, box, x, i, rc2, buf, 0);
        free(buf);
    }
    off[0] = 0;
    for (int i = 0; i < n; i++) off[i + 1] = off[i] + cnt[i];
    int *nbr = (int *)malloc(sizeof(int) * (off[n] > 0 ? off[n] : 1));
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int i = 0; i < n; i++) pairs_row(&g, box, x, i, rc2, nbr + off[i], cnt[i]);
    free(cnt);
    free(g.head); free(g.next);
    *off_out = off;
    *nbr_out = nbr;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Reductions                                                                 */
/* ------------------------------------------------------------------------- */
/* Kahan sum in index order, src/utils/CVs_tools.cu:6-18. */
static double kahan_sum_masked(int n, const double *v, const int *ingroup) {
    double s = 0.0, c = 0.0;
    for (int i = 0; i < n; i++) {
        if (!ingroup[i]) continue;
        double y = v[i] - c, t = s + y;
        c = (t - s) - y;
        s = t;
    }
    return s;
}

static int group_count(int n, const int *ingroup) {
    int c = 0;
    for (int i = 0; i < n; i++) c += ingroup[i] ? 1 : 0;
    return c;
}

/* Per-thread gradient accumulators reduced in thread order. */
static double *grad_buffers(int nth, int n) { return (double *)calloc((size_t)nth * n * 3, sizeof(double)); }
static void grad_reduce(int nth, int n, const double *bufs, double *grad) {
    for (int i = 0; i < 3 * n; i++) {
        double s = 0.0;
        for (int t = 0; t < nth; t++) s += bufs[(size_t)t * n * 3 + i];
        grad[i] = s;
    }
}
static int thread_id(void) {
#ifdef _OPENMP
    return omp_get_thread_num();
#else
    return 0;
#endif
}

/* ------------------------------------------------------------------------- */
/* STEINH Q: src/cvs/CVs_Steinhardt.cu:1324-1532 (values), :825-977 (CV),     */
/* exact gradient in place of :1538-1863                                      */
/* ------------------------------------------------------------------------- */
typedef struct { double r2; int j; } rj;
static int cmp_rj(const void *a, const void *b) {
    const rj *x = (const rj *)a, *y = (const rj *)b;
    if (x->r2 < y->r2) return -1;
    if (x->r2 > y->r2) return 1;
    return (x->j > y->j) - (x->j < y->j);
}

int orc_steinh_q(int l, int n, const double *x, const orc_box *box, const int *ingroup,
                 double rc, int cap, int mode, const orc_sw *swcv,
                 double *Q, double *qlm, int *nkept, int *nrc, int *kept,
                 double *cv, double *grad) {
    init_tables();
    if (l < 1 || l > ORC_LMAX || cap < 1) return 1;
    const int S = 2 * (l + 1);
    const double C = 4.0 * ORC_PI / (2.0 * l + 1.0);
    int64_t *off; int *nbr;
    orc_pairs(n, x, box, rc, &off, &nbr);
    double rc2 = rc * rc;
    int nth = orc_get_threads();
#pragma omp parallel num_threads(nth)
    {
        rj *tmp = (rj *)malloc(sizeof(rj) * 4096);
        double yre[ORC_LMAX + 1], yim[ORC_LMAX + 1];
#pragma omp for schedule(static)
        for (int i = 0; i < n; i++) {
            int c = 0;
            for (int64_t p = off[i]; p < off[i + 1]; p++) {
                int j = nbr[p];
                double d[3];
                orc_minimg(box, x + 3 * i, x + 3 * j, d);
                double r2 = orc_r2(d);
                if (r2 > rc2 || r2 < 1e-12) continue;
                if (c < 4096) { tmp[c].r2 = r2; tmp[c].j = j; }
                c++;
            }
            if (c > 4096) c = 4096;
            qsort(tmp, c, sizeof(rj), cmp_rj);
            int k = c < cap ? c : cap;
            nrc[i] = c;
            nkept[i] = k;
            for (int t = 0; t < cap; t++) kept[(int64_t)i * cap + t] = t < k ? tmp[t].j : -1;
            double acc[2 * (ORC_LMAX + 1)];
            memset(acc, 0, sizeof(acc));
            for (int t = 0; t < k; t++) {
                double d[3];
                orc_minimg(box, x + 3 * i, x + 3 * tmp[t].j, d);
                orc_ylm(l, d, yre, yim);
                for (int m = 0; m <= l; m++) { acc[2 * m] += yre[m]; acc[2 * m + 1] += yim[m]; }
            }
            double q2 = 0.0;
            for (int s = 0; s < S; s++) {
                double v = k > 0 ? acc[s] / k : 0.0;
                qlm[(int64_t)i * S + s] = v;
            }
            for (int m = 0; m <= l; m++) {
                double a = qlm[(int64_t)i * S + 2 * m], b = qlm[(int64_t)i * S + 2 * m + 1];
                q2 += (m == 0 ? 1.0 : 2.0) * (a * a + b * b);
            }
            Q[i] = k > 0 ? sqrt(q2 * C) : 0.0;
        }
        free(tmp);
    }
    int N = group_count(n, ingroup);
    double val;
    if (mode == 0) {
        val = (N > 0) ? kahan_sum_masked(n, Q, ingroup) / N : 0.0;
    } else {
        val = 0.0;
        for (int i = 0; i < n; i++) if (ingroup[i]) val += orc_sw_f(swcv, Q[i]);
    }
    *cv = val;
    if (grad) {
        double *bufs = grad_buffers(nth, n);
#pragma omp parallel num_threads(nth)
        {
            double *g = bufs + (size_t)thread_id() * n * 3;
            double yre[ORC_LMAX + 1], yim[ORC_LMAX + 1], gre[3 * (ORC_LMAX + 1)], gim[3 * (ORC_LMAX + 1)];
#pragma omp for schedule(static)
            for (int i = 0; i < n; i++) {
                if (!ingroup[i] || nkept[i] == 0 || Q[i] <= 0.0) continue;
                double dcv = (mode == 0) ? 1.0 / N : orc_sw_df(swcv, Q[i]);
                double a = dcv * C / Q[i] / nkept[i];
                for (int t = 0; t < nkept[i]; t++) {
                    int j = kept[(int64_t)i * cap + t];
                    double d[3];
                    orc_minimg(box, x + 3 * i, x + 3 * j, d);
                    orc_ylm_grad(l, d, yre, yim, gre, gim);
                    double v[3] = {0, 0, 0};
                    for (int m = 0; m <= l; m++) {
                        double w = (m == 0 ? 1.0 : 2.0) * a;
                        double lr = w * qlm[(int64_t)i * S + 2 * m], li = w * qlm[(int64_t)i * S + 2 * m + 1];
                        for (int c = 0; c < 3; c++) v[c] += lr * gre[3 * m + c] + li * gim[3 * m + c];
                    }
                    for (int c = 0; c < 3; c++) { g[3 * j + c] += v[c]; g[3 * i + c] -= v[c]; }
                }
            }
        }
        grad_reduce(nth, n, bufs, grad);
        free(bufs);
    }
    free(off); free(nbr);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* STEINH L: src/cvs/CVs_Steinhardt_Local.cu:1210-1580 (values),              */
/* :695-745 (CV), :1622-2130 (gradient; restated from its exact derivation)   */
/* ------------------------------------------------------------------------- */
/* The neighbour lists orc_steinh_l uses: j != i with r <= rlist and
 * sigma(r) >= eps (Local.cu:1257-1262), CSR with j ascending.  Caller frees
 * *off and *nbr with orc_free. */
int orc_local_lists(int n, const double *x, const orc_box *box, double rlist, const orc_sw *swr, double eps,
                    int64_t **off_out, int **nbr_out) {
    int64_t *off; int *nbr;
    orc_pairs(n, x, box, rlist, &off, &nbr);
    int64_t *o2 = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int *n2 = (int *)malloc(sizeof(int) * (size_t)(off[n] > 0 ? off[n] : 1));
    o2[0] = 0;
    for (int i = 0; i < n; i++) {
        int64_t c = o2[i];
        for (int64_t p = off[i]; p < off[i + 1]; p++) {
            double d[3];
            orc_minimg(box, x + 3 * i, x + 3 * nbr[p], d);
            if (orc_sw_f(swr, sqrt(orc_r2(d))) >= eps) n2[c++] = nbr[p];
        }
        o2[i + 1] = c;
    }
    free(off);
    free(nbr);
    *off_out = o2;
    *nbr_out = n2;
    return 0;
}

int orc_steinh_l(int l, int n, const double *x, const orc_box *box, const int *ingroup,
                 double rlist, const orc_sw *swr, double eps, const orc_sw *swcv, int mode,
                 double *LQ, double *LQlm, double *qlm, double *NF, int *nnb,
                 double *cv, double *sums, double *grad) {
    init_tables();
    if (l < 1 || l > ORC_LMAX) return 1;
    const int S = 2 * (l + 1);
    const double C = 4.0 * ORC_PI / (2.0 * l + 1.0);
    int64_t *off; int *nbr;
    orc_pairs(n, x, box, rlist, &off, &nbr);
    int nth = orc_get_threads();
    /* neighbour filter sigma(r) >= eps (Local.cu:1257-1262) */
    int64_t np = off[n];
    double *sig = (double *)malloc(sizeof(double) * (np > 0 ? np : 1));
    char *keep = (char *)malloc(np > 0 ? np : 1);
    int *active = (int *)calloc(n > 0 ? n : 1, sizeof(int));
#pragma omp parallel num_threads(nth)
    {
        double yre[ORC_LMAX + 1], yim[ORC_LMAX + 1];
#pragma omp for schedule(static)
        for (int i = 0; i < n; i++) {
            double nf = 0.0, acc[2 * (ORC_LMAX + 1)];
            int c = 0;
            memset(acc, 0, sizeof(acc));
            for (int64_t p = off[i]; p < off[i + 1]; p++) {
                double d[3];
                orc_minimg(box, x + 3 * i, x + 3 * nbr[p], d);
                double r = sqrt(orc_r2(d));
                double s = orc_sw_f(swr, r);
                sig[p] = s;
                keep[p] = (s >= eps);
                if (!keep[p]) continue;
                nf += s;
                c++;
                orc_ylm(l, d, yre, yim);
                for (int m = 0; m <= l; m++) { acc[2 * m] += s * yre[m]; acc[2 * m + 1] += s * yim[m]; }
            }
            nnb[i] = c;
            NF[i] = nf;
            active[i] = (c > 0 && nf >= 1e-12);
            for (int s = 0; s < S; s++) qlm[(int64_t)i * S + s] = active[i] ? acc[s] / nf : 0.0;
        }
    }
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int i = 0; i < n; i++) {
        double A[2 * (ORC_LMAX + 1)];
        if (!ingroup[i] || !active[i]) {
            for (int s = 0; s < S; s++) LQlm[(int64_t)i * S + s] = 0.0;
            LQ[i] = 0.0;
            continue;
        }
        for (int s = 0; s < S; s++) A[s] = qlm[(int64_t)i * S + s];
        for (int64_t p = off[i]; p < off[i + 1]; p++) {
            if (!keep[p]) continue;
            int j = nbr[p];
            for (int s = 0; s < S; s++) A[s] += sig[p] * qlm[(int64_t)j * S + s];
        }
        double q2 = 0.0;
        for (int s = 0; s < S; s++) LQlm[(int64_t)i * S + s] = A[s] / (NF[i] + 1.0);
        for (int m = 0; m <= l; m++) {
            double a = LQlm[(int64_t)i * S + 2 * m], b = LQlm[(int64_t)i * S + 2 * m + 1];
            q2 += (m == 0 ? 1.0 : 2.0) * (a * a + b * b);
        }
        LQ[i] = sqrt(q2 * C);
    }
    /* reductions, Kahan in index order: src/utils/CVs_tools.cu:20-55 */
    double s1 = 0, c1 = 0, s0 = 0, c0 = 0;
    for (int i = 0; i < n; i++) {
        if (!ingroup[i]) continue;
        double w = orc_sw_f(swcv, LQ[i]);
        double y = w - c0, t = s0 + y; c0 = (t - s0) - y; s0 = t;
        double wv = LQ[i] * w;
        y = wv - c1; t = s1 + y; c1 = (t - s1) - y; s1 = t;
    }
    int N = group_count(n, ingroup);
    sums[0] = s1; sums[1] = s0; sums[2] = N;
    double val;
    if (mode == 0) val = (s0 != 0.0) ? s1 / s0 : 0.0;
    else if (mode == 1) val = s0;
    else val = (N > 0) ? s0 / (double)N : 0.0;
    *cv = val;
    if (grad) {
        /* adjoint of A_i: G_i = F_i w_m LQlm_i / (NF_i + 1) */
        double *G = (double *)calloc((size_t)n * S, sizeof(double));
        double *lam = (double *)calloc((size_t)n * S, sizeof(double));
        for (int i = 0; i < n; i++) {
            if (!ingroup[i] || !active[i]) continue;
            double lq = LQ[i] > 1e-12 ? LQ[i] : 1e-12;
            double dcv;
            if (mode == 0) {
                double W = s0 > 1e-300 ? s0 : 1e-300;
                dcv = (orc_sw_df(swcv, LQ[i]) * (LQ[i] - val) + orc_sw_f(swcv, LQ[i])) / W;
            } else if (mode == 1) dcv = orc_sw_df(swcv, LQ[i]);
            else dcv = orc_sw_df(swcv, LQ[i]) / (N > 1 ? (double)N : 1.0);
            double F = dcv * C / lq / (NF[i] + 1.0);
            for (int m = 0; m <= l; m++) {
                double w = (m == 0 ? 1.0 : 2.0) * F;
                G[(int64_t)i * S + 2 * m] = w * LQlm[(int64_t)i * S + 2 * m];
                G[(int64_t)i * S + 2 * m + 1] = w * LQlm[(int64_t)i * S + 2 * m + 1];
            }
        }
        /* lambda_k = G_k + sum_{i: k in N(i)} sigma_ik G_i  (serial scatter) */
        for (int i = 0; i < n; i++) {
            if (!ingroup[i] || !active[i]) continue;
            for (int s = 0; s < S; s++) lam[(int64_t)i * S + s] += G[(int64_t)i * S + s];
            for (int64_t p = off[i]; p < off[i + 1]; p++) {
                if (!keep[p]) continue;
                int j = nbr[p];
                for (int s = 0; s < S; s++) lam[(int64_t)j * S + s] += sig[p] * G[(int64_t)i * S + s];
            }
        }
        double *bufs = grad_buffers(nth, n);
#pragma omp parallel num_threads(nth)
        {
            double *g = bufs + (size_t)thread_id() * n * 3;
            double yre[ORC_LMAX + 1], yim[ORC_LMAX + 1], gre[3 * (ORC_LMAX + 1)], gim[3 * (ORC_LMAX + 1)];
#pragma omp for schedule(static)
            for (int i = 0; i < n; i++) {
                if (!active[i]) continue;
                int gi = ingroup[i];
                for (int64_t p = off[i]; p < off[i + 1]; p++) {
                    if (!keep[p]) continue;
                    int j = nbr[p];
                    double d[3];
                    orc_minimg(box, x + 3 * i, x + 3 * j, d);
                    double r = sqrt(orc_r2(d));
                    double dsig = orc_sw_df(swr, r);
                    double v[3] = {0, 0, 0};
                    orc_ylm_grad(l, d, yre, yim, gre, gim);
                    /* (i,j) LQ term: dsigma_ij * Re(G_i . (q_j - LQlm_i)) */
                    double coef = 0.0;
                    if (gi && dsig != 0.0)
                        for (int s = 0; s < S; s++)
                            coef += G[(int64_t)i * S + s] * (qlm[(int64_t)j * S + s] - LQlm[(int64_t)i * S + s]);
                    /* (i,j) q term: [dsigma Re(lam.(Y - q_i)) + sigma Re(lam . dY)] / NF_i */
                    double cy = 0.0;
                    for (int m = 0; m <= l; m++) {
                        double lr = lam[(int64_t)i * S + 2 * m], li = lam[(int64_t)i * S + 2 * m + 1];
                        cy += lr * (yre[m] - qlm[(int64_t)i * S + 2 * m]) + li * (yim[m] - qlm[(int64_t)i * S + 2 * m + 1]);
                        for (int c = 0; c < 3; c++)
                            v[c] += sig[p] / NF[i] * (lr * gre[3 * m + c] + li * gim[3 * m + c]);
                    }
                    double radial = dsig * (coef + cy / NF[i]) / r;
                    for (int c = 0; c < 3; c++) v[c] += radial * d[c];
                    for (int c = 0; c < 3; c++) { g[3 * j + c] += v[c]; g[3 * i + c] -= v[c]; }
                }
            }
        }
        grad_reduce(nth, n, bufs, grad);
        free(bufs);
        free(G); free(lam);
    }
    free(sig); free(keep); free(active);
    free(off); free(nbr);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* STRU_FACTOR, Debye form: src/cvs/CVs_Strufactor.cu:1014-1271               */
/* ------------------------------------------------------------------------- */
static void debye_g(double r2, double rc2, double qf, double *g, double *dg) {
    double r = sqrt(r2), th = qf * r, s = 1.0, ds = 0.0;
    double r_on = 0.8 * rc2;
    if (r2 > r_on) {
        double t = (r2 - r_on) / (rc2 - r_on);
        s = 1.0 - t * t * t;
        ds = -3.0 * t * t * (2.0 * r) / (rc2 - r_on);
    }
    if (qf == 0.0) {   /* WEIGHT_CHEM pair term (CV_Weighted_Chemical_Pair_Order.cu:647-690) */
        *g = s;
        *dg = ds;
        return;
    }
    double sn = sin(th), cs = cos(th);
    *g = sn / th * s;
    *dg = (cs / th - sn / (th * th)) * s * qf + ds * sn / th;
}

int orc_debye(int n, const double *x, const orc_box *box, const int *ingroup,
              double rc, double qf, int mode, const orc_sw *sw,
              double *S, double *cv, double *grad) {
    return orc_debye_w(n, x, box, ingroup, rc, qf, mode, sw, NULL, S, cv, grad);
}

/* STRU_FACTOR Chemical (src/cvs/CVs_Strufactor_chem.cu:137-175, :204-265): every
 * pair term times w_i w_j, the per-atom type weights (w = NULL: all 1). */
int orc_debye_w(int n, const double *x, const orc_box *box, const int *ingroup,
                double rc, double qf, int mode, const orc_sw *sw, const double *w,
                double *S, double *cv, double *grad) {
    int64_t *off; int *nbr;
    orc_pairs(n, x, box, rc, &off, &nbr);
    double rc2 = rc * rc;
    int nth = orc_get_threads();
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int i = 0; i < n; i++) {
        if (!ingroup[i]) { S[i] = 0.0; continue; }
        double acc = 0.0;
        for (int64_t p = off[i]; p < off[i + 1]; p++) {
            double d[3];
            orc_minimg(box, x + 3 * i, x + 3 * nbr[p], d);
            double r2 = orc_r2(d);
            if (r2 > rc2 || r2 < 1e-12) continue;
            double g, dg;
            debye_g(r2, rc2, qf, &g, &dg);
            acc += w ? w[i] * w[nbr[p]] * g : g;
        }
        S[i] = acc + 1.0;
    }
    int N = group_count(n, ingroup);
    double val;
    if (mode == 0) val = N > 0 ? kahan_sum_masked(n, S, ingroup) / N : 0.0;
    else { val = 0.0; for (int i = 0; i < n; i++) if (ingroup[i]) val += orc_sw_f(sw, S[i]); }
    *cv = val;
    if (grad) {
        double *bufs = grad_buffers(nth, n);
#pragma omp parallel num_threads(nth)
        {
            double *g = bufs + (size_t)thread_id() * n * 3;
#pragma omp for schedule(static)
            for (int i = 0; i < n; i++) {
                if (!ingroup[i]) continue;
                double a = (mode == 0) ? 1.0 / N : orc_sw_df(sw, S[i]);
                for (int64_t p = off[i]; p < off[i + 1]; p++) {
                    int j = nbr[p];
                    double d[3];
                    orc_minimg(box, x + 3 * i, x + 3 * j, d);
                    double r2 = orc_r2(d);
                    if (r2 > rc2 || r2 < 1e-12) continue;
                    double gv, dg;
                    debye_g(r2, rc2, qf, &gv, &dg);
                    double r = sqrt(r2);
                    double aw = w ? a * w[i] * w[j] : a;
                    for (int c = 0; c < 3; c++) { double v = aw * dg * d[c] / r; g[3 * j + c] += v; g[3 * i + c] -= v; }
                }
            }
        }
        grad_reduce(nth, n, bufs, grad);
        free(bufs);
    }
    free(off); free(nbr);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* k-vector S(k) (no reference counterpart)                                    */
/* ------------------------------------------------------------------------- */
int orc_sk(int n, const double *x, const int *ingroup, int nk, const double *k,
           double *rho, double *Sk, double *cv, double *grad) {
    int N = group_count(n, ingroup);
    int nth = orc_get_threads();
    double acc_cv = 0.0;
    for (int q = 0; q < nk; q++) {
        double re = 0.0, im = 0.0;
#pragma omp parallel for reduction(+ : re, im) schedule(static) num_threads(nth)
        for (int i = 0; i < n; i++) {
            if (!ingroup[i]) continue;
            double ph = k[3 * q] * x[3 * i] + k[3 * q + 1] * x[3 * i + 1] + k[3 * q + 2] * x[3 * i + 2];
            re += cos(ph);
            im += sin(ph);
        }
        rho[2 * q] = re; rho[2 * q + 1] = im;
        Sk[q] = N > 0 ? (re * re + im * im) / N : 0.0;
        acc_cv += Sk[q];
    }
    *cv = nk > 0 ? acc_cv / nk : 0.0;
    if (grad) {
#pragma omp parallel for schedule(static) num_threads(nth)
        for (int i = 0; i < n; i++) {
            double g[3] = {0, 0, 0};
            if (ingroup[i] && N > 0) {
                for (int q = 0; q < nk; q++) {
                    double ph = k[3 * q] * x[3 * i] + k[3 * q + 1] * x[3 * i + 1] + k[3 * q + 2] * x[3 * i + 2];
                    double a = (2.0 / N) * (-rho[2 * q] * sin(ph) + rho[2 * q + 1] * cos(ph));
                    for (int c = 0; c < 3; c++) g[c] += a * k[3 * q + c];
                }
                for (int c = 0; c < 3; c++) g[c] /= nk;
            }
            for (int c = 0; c < 3; c++) grad[3 * i + c] = g[c];
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Bias grid: src/grids/GH_t0_uniformGrid.cu                                  */
/* ------------------------------------------------------------------------- */
static double cr_value(double p0, double p1, double p2, double p3, double x) {   /* :289-295 */
    return p1 + 0.5 * x * ((p2 - p0) + x * (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3) + x * x * (-p0 + 3.0 * p1 - 3.0 * p2 + p3));
}
static double cr_deriv(double p0, double p1, double p2, double p3, double x) {   /* :296-302 */
    return 0.5 * ((p2 - p0) + 2.0 * x * (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3) + 3.0 * x * x * (-p0 + 3.0 * p1 - 3.0 * p2 + p3));
}
static void center_frac_clamp(double cv, double lo, double h, int nb, int *i, double *f) {   /* :304-310 */
    double u = (cv - lo) / h - 0.5;
    int k = (int)floor(u);
    double fr = u - k;
    if (k < 1) { k = 1; fr = 0.0; }
    if (k > nb - 3) { k = nb - 3; fr = 1.0; }
    *i = k; *f = fr;
}

/* Banded deposit (:227-264).  The band radius uses sigma_band (the fix's sigma,
 * :87), the Gaussian uses sigma (a restart hill's own sigma, :160). */
void orc_grid_deposit(int D, const int *nbin, const double *bound, double *grid,
                      const double *s, double w, double sigma, double sigma_band) {
    double dcv[3];
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    for (int k = 0; k < D; k++) {
        dcv[k] = (bound[2 * k + 1] - bound[2 * k]) / nbin[k];
        int R = (int)ceil(4.0 * sigma_band / dcv[k]) + 1;
        double u = (s[k] - bound[2 * k]) / dcv[k];
        /* a centre far outside the grid (or not finite) leaves the band empty, as the
         * reference's lower > upper loops do, without the int overflow of a huge cast */
        if (!(u > -(double)R - 2.0 && u < (double)nbin[k] + R + 2.0)) return;
        int c = (int)u;
        lo[k] = c - R < 0 ? 0 : c - R;
        hi[k] = c + R > nbin[k] - 1 ? nbin[k] - 1 : c + R;
    }
    double s2 = sigma * sigma;
    if (D == 1) {
        for (long g = lo[0]; g <= hi[0]; g++) {
            double dx = s[0] - (bound[0] + (g + 0.5) * (bound[1] - bound[0]) / nbin[0]);
            grid[g] += w * exp(-0.5 * (dx * dx) / s2);
        }
    } else if (D == 2) {
        for (long i = lo[0]; i <= hi[0]; i++)
            for (long j = lo[1]; j <= hi[1]; j++) {
                double dx = s[0] - (bound[0] + (i + 0.5) * (bound[1] - bound[0]) / nbin[0]);
                double dy = s[1] - (bound[2] + (j + 0.5) * (bound[3] - bound[2]) / nbin[1]);
                grid[i * nbin[1] + j] += w * exp(-0.5 * (dx * dx + dy * dy) / s2);
            }
    } else {
        for (long i = lo[0]; i <= hi[0]; i++)
            for (long j = lo[1]; j <= hi[1]; j++)
                for (long k = lo[2]; k <= hi[2]; k++) {
                    double dx = s[0] - (bound[0] + (i + 0.5) * (bound[1] - bound[0]) / nbin[0]);
                    double dy = s[1] - (bound[2] + (j + 0.5) * (bound[3] - bound[2]) / nbin[1]);
                    double dz = s[2] - (bound[4] + (k + 0.5) * (bound[5] - bound[4]) / nbin[2]);
                    grid[(i * nbin[1] + j) * nbin[2] + k] += w * exp(-0.5 * (dx * dx + dy * dy + dz * dz) / s2);
                }
    }
}

double orc_grid_value(int D, const int *nbin, const double *bound, const double *grid,
                      const double *s, double *dVds) {
    int ix[3]; double fx[3], dcv[3];
    for (int k = 0; k < D; k++) {
        dcv[k] = (bound[2 * k + 1] - bound[2 * k]) / nbin[k];
        center_frac_clamp(s[k], bound[2 * k], dcv[k], nbin[k], &ix[k], &fx[k]);
    }
    double V;
    if (D == 1) {
        const double *p = grid + ix[0] - 1;
        V = cr_value(p[0], p[1], p[2], p[3], fx[0]);
        dVds[0] = cr_deriv(p[0], p[1], p[2], p[3], fx[0]) / dcv[0];
        if (isnan(dVds[0])) dVds[0] = 0.0;
    } else if (D == 2) {
        double col[4], dcol[4];
        int n1 = nbin[1];
        for (int t = 0; t < 4; t++) {
            int jj = ix[1] - 1 + t;
            double p0 = grid[(ix[0] - 1) * n1 + jj], p1 = grid[ix[0] * n1 + jj];
            double p2 = grid[(ix[0] + 1) * n1 + jj], p3 = grid[(ix[0] + 2) * n1 + jj];
            col[t] = cr_value(p0, p1, p2, p3, fx[0]);
            dcol[t] = cr_deriv(p0, p1, p2, p3, fx[0]);
        }
        V = cr_value(col[0], col[1], col[2], col[3], fx[1]);
        dVds[0] = cr_value(dcol[0], dcol[1], dcol[2], dcol[3], fx[1]) / dcv[0];
        dVds[1] = cr_deriv(col[0], col[1], col[2], col[3], fx[1]) / dcv[1];
        if (isnan(dVds[0]) || isnan(dVds[1])) { dVds[0] = 0.0; dVds[1] = 0.0; }
    } else {
        /* tricubic: dim 0 innermost, then dim 1, then dim 2 */
        int n1 = nbin[1], n2 = nbin[2];
        double a[4], da[4], b0[4], b1[4], b2[4];
        for (int u = 0; u < 4; u++) {
            int kk = ix[2] - 1 + u;
            double c[4], dc[4];
            for (int t = 0; t < 4; t++) {
                int jj = ix[1] - 1 + t;
                double p[4];
                for (int q = 0; q < 4; q++) p[q] = grid[((ix[0] - 1 + q) * n1 + jj) * n2 + kk];
                c[t] = cr_value(p[0], p[1], p[2], p[3], fx[0]);
                dc[t] = cr_deriv(p[0], p[1], p[2], p[3], fx[0]);
            }
            a[u] = cr_value(c[0], c[1], c[2], c[3], fx[1]);
            da[u] = cr_deriv(c[0], c[1], c[2], c[3], fx[1]);
            b0[u] = cr_value(dc[0], dc[1], dc[2], dc[3], fx[1]);
            (void)b1; (void)b2;
        }
        V = cr_value(a[0], a[1], a[2], a[3], fx[2]);
        dVds[0] = cr_value(b0[0], b0[1], b0[2], b0[3], fx[2]) / dcv[0];
        dVds[1] = cr_value(da[0], da[1], da[2], da[3], fx[2]) / dcv[1];
        dVds[2] = cr_deriv(a[0], a[1], a[2], a[3], fx[2]) / dcv[2];
        if (isnan(dVds[0]) || isnan(dVds[1]) || isnan(dVds[2])) { dVds[0] = dVds[1] = dVds[2] = 0.0; }
    }
    return V;
}

void orc_hill_sum(int D, int nh, const double *centers, const double *heights, const double *sigmas,
                  int np, const double *points, double *V, double *dV) {
    int nth = orc_get_threads();
#pragma omp parallel for schedule(static) num_threads(nth)
    for (int p = 0; p < np; p++) {
        double v = 0.0, g[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int h = 0; h < nh; h++) {
            double r2 = 0.0, dd[8];
            for (int k = 0; k < D; k++) { dd[k] = points[p * D + k] - centers[h * D + k]; r2 += dd[k] * dd[k]; }
            double s2 = sigmas[h] * sigmas[h];
            double e = heights[h] * exp(-0.5 * r2 / s2);
            v += e;
            for (int k = 0; k < D; k++) g[k] -= e * dd[k] / s2;
        }
        V[p] = v;
        if (dV) for (int k = 0; k < D; k++) dV[p * D + k] = g[k];
    }
}
