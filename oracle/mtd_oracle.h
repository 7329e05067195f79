/*
 * mtd_oracle.h -- CPU FP64 restatement of the Metad-toy metadynamics hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle for the
 * sm_100a product in metad-toy_b200/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it.  The product never links it.
 *
 * Every routine cites the reference file:line whose behaviour it restates
 * (paths relative to the Metad-toy project root).  Where the reference is
 * mathematically wrong the oracle computes the exact quantity and says so.
 */
#ifndef MTD_ORACLE_H
#define MTD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Switching function, restates include/utils/zqc_switch_function.h:16-31. */
typedef struct {
    int type;          /* 0 LINE, 1 STEP, 2 FERMI, 3 TANH, 4 RATIONAL */
    double r0, d0, alpha;
    int n, m;
} orc_sw;

typedef struct {
    double L[3];       /* box lengths */
    int periodic[3];
} orc_box;

double orc_sw_f(const orc_sw *p, double x);
double orc_sw_df(const orc_sw *p, double x);
double orc_sw_invert_for_eps(const orc_sw *p, double eps);

/* Spherical harmonics (complex, orthonormal, Condon-Shortley phase), m = 0..l.
 * Restates the closed forms of include/CVsets/CV_Steinhardt_math.h:981-1217
 * by the associated-Legendre definition instead of the generated formulas. */
void orc_ylm(int l, const double d[3], double *yre, double *yim);
/* Y_lm and its gradient with respect to the displacement d (not the unit vector).
 * g*[m*3 + c] = dY_lm / d d_c. */
void orc_ylm_grad(int l, const double d[3], double *yre, double *yim, double *gre, double *gim);

/* Minimum-image displacement x_j - x_i, restating the ghost-atom displacement
 * of src/cvs/CVs_Steinhardt.cu:1352-1357 for a single periodic image. */
void orc_minimg(const orc_box *b, const double *xi, const double *xj, double *d);
double orc_r2(const double *d);

/* All ordered pairs (i, j != i) with r2 <= rcut^2, CSR, j ascending.
 * Caller frees *off and *nbr with orc_free. Returns 0 on success. */
int orc_pairs(int n, const double *x, const orc_box *box, double rcut, int64_t **off, int **nbr);
void orc_free(void *p);

/* STEINH Q: cap-N nearest neighbours within rc (r2 <= rc^2, r2 >= 1e-12), ties by
 * (r2, index); q_lm mean; Q_l; CV AVE (Kahan mean over group, restates
 * src/utils/CVs_tools.cu:6-18) or SW_FUNC (sum of f(Q) over group,
 * src/cvs/CVs_Steinhardt.cu:961-977).  grad = exact dCV/dx (n*3), may be NULL.
 * kept: n*cap neighbour indices in (r2, index) order, -1 padded. */
int orc_steinh_q(int l, int n, const double *x, const orc_box *box, const int *ingroup,
                 double rc, int cap, int mode, const orc_sw *swcv,
                 double *Q, double *qlm, int *nkept, int *nrc, int *kept,
                 double *cv, double *grad);

/* STEINH L (local-averaged Q_l): neighbours j != i with r <= rlist and
 * sigma(r) >= eps; q_lm weighted by sigma / NF; LQ_lm = (q_i + sum sigma q_j)/(NF+1).
 * mode 0 MEAN_SOLID, 1 NSOLID, 2 FRAC (src/cvs/CVs_Steinhardt_Local.cu:695-745).
 * sums[0] = sum LQ f(LQ), sums[1] = sum f(LQ), sums[2] = group count. */
int orc_steinh_l(int l, int n, const double *x, const orc_box *box, const int *ingroup,
                 double rlist, const orc_sw *swr, double eps, const orc_sw *swcv, int mode,
                 double *LQ, double *LQlm, double *qlm, double *NF, int *nnb,
                 double *cv, double *sums, double *grad);

/* The lists of orc_steinh_l: j != i, r <= rlist, sigma(r) >= eps; CSR, j ascending. */
int orc_local_lists(int n, const double *x, const orc_box *box, double rlist, const orc_sw *swr, double eps,
                    int64_t **off, int **nbr);

/* STRU_FACTOR (Debye form): S_i = 1 + sum_j sin(q r)/(q r) s(r), r2 in [1e-12, rc^2].
 * mode 0 AVE, 1 COUNT (src/cvs/CVs_Strufactor.cu:642-674, :1082-1271). */
int orc_debye(int n, const double *x, const orc_box *box, const int *ingroup,
              double rc, double qf, int mode, const orc_sw *sw,
              double *S, double *cv, double *grad);
int orc_debye_w(int n, const double *x, const orc_box *box, const int *ingroup,
                double rc, double qf, int mode, const orc_sw *sw, const double *w,
                double *S, double *cv, double *grad);

/* k-vector structure factor: rho_k = sum_{j in group} exp(i k.x_j), S(k) = |rho_k|^2/N,
 * CV = mean_k S(k).  No reference counterpart. */
int orc_sk(int n, const double *x, const int *ingroup, int nk, const double *k,
           double *rho, double *Sk, double *cv, double *grad);

/* Uniform bias grid, restates src/grids/GH_t0_uniformGrid.cu:74-485 for D = 1..3
 * (3D made consistent with 1D/2D: banded deposit and tricubic Catmull-Rom). */
void orc_grid_deposit(int D, const int *nbin, const double *bound, double *grid,
                      const double *s, double w, double sigma, double sigma_band);
double orc_grid_value(int D, const int *nbin, const double *bound, const double *grid,
                      const double *s, double *dVds);

/* Exact FP64 hill sum V(s) = sum_h w_h exp(-|s - c_h|^2 / (2 sigma_h^2)) and dV/ds. */
void orc_hill_sum(int D, int nh, const double *centers, const double *heights, const double *sigmas,
                  int np, const double *points, double *V, double *dV);

void orc_set_threads(int nthreads);
int orc_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
