// bias.cu -- the per-step bias kernel: global CV reductions, DIM expressions,
// well-tempered hill deposit on the FP64 grid, Catmull-Rom V(s) and dV/ds, and
// the chain-rule coefficients handed to the force kernels.  One block; the
// step number is a kernel argument so no host round trip is needed.
//
// Replaces, on the device:
//   KahanAverager / compute_sw reductions   src/utils/CVs_tools.cu:6-55
//   MetaDimensionManager::compute_*          src/grids/DimSet.cu:68-97
//   GH_t0_uniformGrid::add_hill/add_to_grid  src/grids/GH_t0_uniformGrid.cu:195-282
//   GH_t0_uniformGrid::get_dVdcv/get_bias_energy  :313-461
// Built with -fmad=false so the deposit's bin-centre and Gaussian arithmetic
// rounds like the FP64 oracle.
#include "kernels.h"

namespace mtd {

namespace {

__device__ __forceinline__ double cr_value(double p0, double p1, double p2, double p3, double x) {
    return p1 + 0.5 * x * ((p2 - p0) + x * (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3) + x * x * (-p0 + 3.0 * p1 - 3.0 * p2 + p3));
}
__device__ __forceinline__ double cr_deriv(double p0, double p1, double p2, double p3, double x) {
    return 0.5 * ((p2 - p0) + 2.0 * x * (2.0 * p0 - 5.0 * p1 + 4.0 * p2 - p3) + 3.0 * x * x * (-p0 + 3.0 * p1 - 3.0 * p2 + p3));
}
__device__ __forceinline__ void center_frac_clamp(double cv, double lo, double h, int nb, int &i, double &f) {
    double u = (cv - lo) / h - 0.5;
    i = (int)floor(u);
    f = u - i;
    if (i < 1) { i = 1; f = 0.0; }
    if (i > nb - 3) { i = nb - 3; f = 1.0; }
}

// Catmull-Rom stencil of s: base indices ix (clamped) and fractions fx.
__device__ __forceinline__ void stencil_locate(const BiasPlan &P, const double *s, int *ix, double *fx) {
    for (int k = 0; k < P.D; ++k) center_frac_clamp(s[k], P.lo[k], P.dcv[k], P.nbin[k], ix[k], fx[k]);
}

// The 4^D grid values around the stencil, loaded by all threads at once into
// S[((u * 4) + t) * 4 + q] = grid[ix0 - 1 + q][ix1 - 1 + t][ix2 - 1 + u].
__device__ __forceinline__ void stencil_load(const BiasPlan &P, const int *ix, double *S) {
    const int nst = P.D == 1 ? 4 : (P.D == 2 ? 16 : 64);
    for (int e = threadIdx.x; e < nst; e += blockDim.x) {
        const int q = e & 3, t = (e >> 2) & 3, u = e >> 4;
        size_t g = (size_t)(ix[0] - 1 + q);
        if (P.D >= 2) g = g * P.nbin[1] + (ix[1] - 1 + t);
        if (P.D >= 3) g = g * P.nbin[2] + (ix[2] - 1 + u);
        S[e] = __ldcg(P.grid + g);   // through L2: other blocks may have deposited since this SM last read it
    }
}

// Catmull-Rom value and gradient on the bin-centred grid (dimension 0 slowest)
// from a loaded stencil, with the stencil rows spread over threads (all
// threads of the block call it): rows along dimension 0 first, then the
// combination along dimensions 1 and 2 (tensor product, dimension 0 inner).
// Ends synchronised.
__device__ void grid_value_block(const BiasPlan &P, const double *S, const double *fx, double (*row)[16],
                                 double *V, double *dV) {
    const int nrow = P.D == 1 ? 1 : (P.D == 2 ? 4 : 16);
    if (threadIdx.x < nrow) {
        const double *p = S + 4 * threadIdx.x;
        row[0][threadIdx.x] = cr_value(p[0], p[1], p[2], p[3], fx[0]);
        row[1][threadIdx.x] = cr_deriv(p[0], p[1], p[2], p[3], fx[0]);
    }
    __syncthreads();
    if (P.D == 3 && threadIdx.x < 4) {
        const int u = threadIdx.x;
        const double *c = row[0] + 4 * u, *dc = row[1] + 4 * u;
        const double a = cr_value(c[0], c[1], c[2], c[3], fx[1]);
        const double da = cr_deriv(c[0], c[1], c[2], c[3], fx[1]);
        const double b0 = cr_value(dc[0], dc[1], dc[2], dc[3], fx[1]);
        row[2][u] = a;
        row[2][4 + u] = da;
        row[2][8 + u] = b0;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (P.D == 1) {
            *V = row[0][0];
            dV[0] = row[1][0] / P.dcv[0];
            if (isnan(dV[0])) dV[0] = 0.0;
        } else if (P.D == 2) {
            const double *col = row[0], *dcol = row[1];
            *V = cr_value(col[0], col[1], col[2], col[3], fx[1]);
            dV[0] = cr_value(dcol[0], dcol[1], dcol[2], dcol[3], fx[1]) / P.dcv[0];
            dV[1] = cr_deriv(col[0], col[1], col[2], col[3], fx[1]) / P.dcv[1];
            if (isnan(dV[0]) || isnan(dV[1])) { dV[0] = 0.0; dV[1] = 0.0; }
        } else {
            const double *a = row[2], *da = row[2] + 4, *b0 = row[2] + 8;
            *V = cr_value(a[0], a[1], a[2], a[3], fx[2]);
            dV[0] = cr_value(b0[0], b0[1], b0[2], b0[3], fx[2]) / P.dcv[0];
            dV[1] = cr_value(da[0], da[1], da[2], da[3], fx[2]) / P.dcv[1];
            dV[2] = cr_deriv(a[0], a[1], a[2], a[3], fx[2]) / P.dcv[2];
            if (isnan(dV[0]) || isnan(dV[1]) || isnan(dV[2])) dV[0] = dV[1] = dV[2] = 0.0;
        }
    }
    __syncthreads();
}

// Band of a hill: [c - R, c + R] clipped to the grid, c = (int)((s - lo)/dcv)
// (C truncation as in add_to_grid), R from the fix's sigma.  A centre outside
// the grid by more than R bins (or not finite) gives an empty band, which is
// what the reference's `for (g = lower; g <= upper; ...)` loops do.
__device__ __forceinline__ bool hill_band(const BiasPlan &P, const double *s, int *lo, int *hi) {
    bool nonempty = true;
    for (int k = 0; k < P.D; ++k) {
        const double u = (s[k] - P.lo[k]) / P.dcv[k];
        if (!(u > -(double)P.band[k] - 2.0 && u < (double)P.nbin[k] + (double)P.band[k] + 2.0)) {
            lo[k] = 0;
            hi[k] = -1;
            nonempty = false;
            continue;
        }
        const int c = (int)u;
        lo[k] = max(0, c - P.band[k]);
        hi[k] = min(P.nbin[k] - 1, c + P.band[k]);
        if (lo[k] > hi[k]) nonempty = false;
    }
    return nonempty;
}

__device__ __forceinline__ double hill_gauss(const BiasPlan &P, const double *s, const int *idx, double sigma) {
    double r2 = 0.0;
    for (int k = 0; k < P.D; ++k) {
        const double c = P.lo[k] + (idx[k] + 0.5) * (P.hi[k] - P.lo[k]) / P.nbin[k];
        const double dx = s[k] - c;
        r2 = r2 + dx * dx;
    }
    return exp(-0.5 * r2 / (sigma * sigma));
}

struct Dual {
    double v;
    double g[kMaxSymbols];
};

__device__ double eval_code(const ExprInstr *code, int n, const double *sym, int nsym, double *grad) {
    Dual st[kMaxExprStack];
    int sp = 0;
    for (int p = 0; p < n; ++p) {
        const ExprInstr c = code[p];
        if (c.op == EOP_CONST || c.op == EOP_SYM) {
            st[sp].v = (c.op == EOP_CONST) ? c.val : sym[c.arg];
            for (int k = 0; k < nsym; ++k) st[sp].g[k] = (c.op == EOP_SYM && k == c.arg) ? 1.0 : 0.0;
            ++sp;
            continue;
        }
        const int na = expr_arity(c.op);
        double a[3] = {0.0, 0.0, 0.0}, d[3];
        for (int i = 0; i < na; ++i) a[i] = st[sp - na + i].v;
        const double v = expr_apply(c.op, a, d);
        Dual &r = st[sp - na];
        for (int k = 0; k < nsym; ++k) {
            double g = 0.0;   // an operand with a zero partial (an unselected branch) contributes nothing
            for (int i = 0; i < na; ++i)
                if (d[i] != 0.0) g += d[i] * st[sp - na + i].g[k];
            r.g[k] = g;
        }
        r.v = v;
        sp -= na - 1;
    }
    for (int k = 0; k < nsym; ++k) grad[k] = st[0].g[k];
    return st[0].v;
}

// ------------------------------------------------------------------ bias phases
// The per-step work is written as phases over one block of 256 threads so the
// single-context kernel and the multi-walker kernels share it.

// The plan (a few KB in device memory) staged in shared memory by all threads.
__device__ __forceinline__ void stage_plan(const BiasPlan *__restrict__ Pp, unsigned char *plan_raw) {
    static_assert(sizeof(BiasPlan) % 16 == 0, "plan size");
    const double2 *src = reinterpret_cast<const double2 *>(Pp);
    double2 *dst = reinterpret_cast<double2 *>(plan_raw);
    for (int e = threadIdx.x; e < (int)(sizeof(BiasPlan) / 16); e += blockDim.x) dst[e] = src[e];
    __syncthreads();
}

// Deterministic reduction of one unit's block partials (rows of 8 doubles,
// four rows in flight per thread); the totals land in usum_u on thread 0.
__device__ void unit_total(const UnitPlan &U, double *smem, double *usum_u) {
    double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (U.partials && U.pstride != 8) {
        for (int b = threadIdx.x; b < U.nparts; b += blockDim.x)
            for (int t = 0; t < U.nvals && t < 8; ++t) v[t] += U.partials[(size_t)b * U.pstride + t];
    } else if (U.partials) {
        const double4 *rows = reinterpret_cast<const double4 *>(U.partials);
        const double4 zero = make_double4(0.0, 0.0, 0.0, 0.0);
        for (int b0 = 0; b0 < U.nparts; b0 += 4 * blockDim.x) {
            double4 r[8];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int b = b0 + threadIdx.x + q * blockDim.x;
                r[2 * q] = b < U.nparts ? rows[2 * (size_t)b] : zero;
                r[2 * q + 1] = b < U.nparts ? rows[2 * (size_t)b + 1] : zero;
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                v[0] += r[2 * q].x; v[1] += r[2 * q].y; v[2] += r[2 * q].z; v[3] += r[2 * q].w;
                v[4] += r[2 * q + 1].x; v[5] += r[2 * q + 1].y; v[6] += r[2 * q + 1].z; v[7] += r[2 * q + 1].w;
            }
        }
    }
    block_sum<8>(v, smem);
    if (threadIdx.x == 0)
        for (int t = 0; t < 8; ++t) usum_u[t] = t < U.nvals ? v[t] : 0.0;
    __syncthreads();
}

// Phases 1-3: every unit's totals (this context's block partials, or the
// totals over all ranks under domain decomposition), symbol values (one
// thread each), DIM expressions with exact chain factors (one thread per
// dimension).
__device__ void phase_cvs(const BiasPlan &P, double *smem, double (*usum)[8], double *s_sym,
                          double (*s_jac)[kMaxSymbols], double *sv) {
    if (P.gsum) {
        for (int e = threadIdx.x; e < P.nunit * 8; e += blockDim.x) usum[e / 8][e % 8] = P.gsum[e];
        __syncthreads();
    } else {
        for (int u = 0; u < P.nunit; ++u) unit_total(P.unit[u], smem, usum[u]);
    }
    if (threadIdx.x < P.nsym) {
        const int q = threadIdx.x;
        const SymPlan &S = P.sym[q];
        const double *us = usum[S.unit];
        double v = 0.0;
        switch (S.kind) {
        case SYM_Q_AVE: v = us[3] > 0 ? us[0] / us[3] : 0.0; break;
        case SYM_Q_SW: v = us[1 + S.slot]; break;
        case SYM_L_MEAN: v = us[2 * S.slot + 1] != 0.0 ? us[2 * S.slot] / us[2 * S.slot + 1] : 0.0; break;
        case SYM_L_NSOLID: v = us[2 * S.slot + 1]; break;
        case SYM_L_FRAC: v = us[4] > 0 ? us[2 * S.slot + 1] / us[4] : 0.0; break;
        case SYM_SF_AVE: v = us[2] > 0 ? us[0] / us[2] : 0.0; break;
        case SYM_SF_COUNT: v = us[1]; break;
        case SYM_SK_AVE: {
            const UnitPlan &U = P.unit[S.unit];
            const double N = *U.sk_n;
            double acc = 0.0;
            for (int k = 0; k < U.K; ++k) acc += U.rho[2 * k] * U.rho[2 * k] + U.rho[2 * k + 1] * U.rho[2 * k + 1];
            v = (N > 0 && U.K > 0) ? acc / N / U.K : 0.0;
            break;
        }
        }
        s_sym[q] = v;
        P.out[kOutSymOffset + q] = v;
    }
    __syncthreads();
    if (threadIdx.x < P.D) sv[threadIdx.x] = eval_code(P.code[threadIdx.x], P.ncode[threadIdx.x], s_sym, P.nsym,
                                                        s_jac[threadIdx.x]);
    __syncthreads();
}

// Phase 4: well-tempered height from V(s) on the stencil before the deposit.
__device__ double phase_wt_height(const BiasPlan &P, const double *sten, const double *fx, double (*row)[16],
                                  double *s_V, double *s_dV) {
    if (P.wt) grid_value_block(P, sten, fx, row, s_V, s_dV);
    return P.h0 * exp(-(P.wt ? *s_V : 0.0) / (P.temp * P.kb * (P.biasf - 1.0)));
}

// Phase 5: banded deposit of one hill, one thread per band bin; the stencil
// (when given) takes the same increment as the grid (same operands, same
// rounding), so V and dV/ds after the deposit need no second grid read.
__device__ void phase_deposit(const BiasPlan &P, const double *s, double w, const int *ix, double *sten) {
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0}, ext[3] = {1, 1, 1};
    int total = 0;
    if (hill_band(P, s, lo, hi)) {
        total = 1;
        for (int k = 0; k < P.D; ++k) {
            ext[k] = hi[k] - lo[k] + 1;
            total *= ext[k];
        }
    }
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        int idx[3] = {0, 0, 0}, rem = t;
        for (int k = P.D - 1; k >= 0; --k) {
            idx[k] = lo[k] + rem % ext[k];
            rem /= ext[k];
        }
        size_t g = idx[0];
        for (int k = 1; k < P.D; ++k) g = g * P.nbin[k] + idx[k];
        if (g < (size_t)P.grid_size) P.grid[g] += w * hill_gauss(P, s, idx, P.sigma);
    }
    const int nst = P.D == 1 ? 4 : (P.D == 2 ? 16 : 64);
    if (sten && total > 0 && threadIdx.x < nst) {
        const int e = threadIdx.x;
        const int idx[3] = {ix[0] - 1 + (e & 3), ix[1] - 1 + ((e >> 2) & 3), ix[2] - 1 + (e >> 4)};
        bool in = true;
        for (int k = 0; k < P.D; ++k) in = in && idx[k] >= lo[k] && idx[k] <= hi[k];
        if (in) sten[e] += w * hill_gauss(P, s, idx, P.sigma);
    }
}

// A step whose neighbour lists overflowed is repeated by the host: it must
// leave no hill and no bias force behind.
// The four words are loaded together (no short-circuit between volatile
// loads, which would wait for each in turn).
__device__ __forceinline__ bool status_failed(const DevStatus *st) {
    if (!st) return false;
    const unsigned a = *(volatile const unsigned *)&st->overflow, b = *(volatile const unsigned *)&st->bad_pos,
                   c = *(volatile const unsigned *)&st->cand_overflow, d = *(volatile const unsigned *)&st->timeout;
    return (a | b | c | d) != 0u;
}
__device__ __forceinline__ bool step_failed(const BiasPlan &P) { return status_failed(P.status); }

__device__ __forceinline__ void record_hill(const BiasPlan &P, long long step, const double *s, double w) {
    const unsigned long long h = *P.nhills;
    HillRec r;
    r.step = step;
    for (int k = 0; k < kMaxDim; ++k) r.s[k] = k < P.D ? s[k] : 0.0;
    r.w = w;
    r.sigma = P.sigma;
    P.hills[h % (unsigned long long)P.hill_cap] = r;
    *reinterpret_cast<HillRec *>(P.out + kOutHillOffset) = r;
    *P.nhills = h + 1;
}

// Phases 6-7: V and dV/ds on the (post-deposit) stencil, chain rule to every
// symbol, outputs, and the per-unit force coefficients (one thread per unit and
// l slot).
__device__ void phase_coef_from_v(const BiasPlan &P, const double *sv, const double (*s_jac)[kMaxSymbols],
                                  const double (*usum)[8], int dep, const double *s_V, const double *s_dV,
                                  double *s_alpha);
__device__ void phase_unit_coefs(const BiasPlan &P, const double (*usum)[8], const double *s_alpha);

__device__ void phase_coef(const BiasPlan &P, const double *sten, const double *fx, const double *sv,
                           const double (*s_jac)[kMaxSymbols], const double (*usum)[8], int dep, double (*row)[16],
                           double *s_V, double *s_dV, double *s_alpha) {
    grid_value_block(P, sten, fx, row, s_V, s_dV);
    phase_coef_from_v(P, sv, s_jac, usum, dep, s_V, s_dV, s_alpha);
}

// V and dV/ds already in shared memory (all threads call it).
__device__ void phase_coef_from_v(const BiasPlan &P, const double *sv, const double (*s_jac)[kMaxSymbols],
                                  const double (*usum)[8], int dep, const double *s_V, const double *s_dV,
                                  double *s_alpha) {
    if (threadIdx.x < P.nsym) {
        const int q = threadIdx.x;
        double a = 0.0;
        for (int dd = 0; dd < P.D; ++dd) a += s_dV[dd] * s_jac[dd][q];
        s_alpha[q] = a;
    }
    if (threadIdx.x == 32) {
        for (int dd = 0; dd < P.D; ++dd) P.out[dd] = sv[dd];
        P.out[P.D] = *s_V;
        P.out[P.D + 1] = dep ? 1.0 : 0.0;
    }
    __syncthreads();
    phase_unit_coefs(P, usum, s_alpha);
}

// Per-unit force coefficients from the chain factors alpha (one thread per
// unit and l slot); zero on a failed step.
__device__ void phase_unit_coefs(const BiasPlan &P, const double (*usum)[8], const double *s_alpha) {
    if (step_failed(P)) {
        for (int e = threadIdx.x; e < P.nunit * 8; e += blockDim.x) P.unit[e / 8].coef[e % 8] = 0.0;
        return;
    }
    if (threadIdx.x < 2 * P.nunit) {
        const int u = threadIdx.x >> 1, slot = threadIdx.x & 1;
        const UnitPlan &U = P.unit[u];
        const double *us = usum[u];
        if (U.kind == 1) {   // STEINH L: c1 = aM/W, c2 = -aM cv/W + aN + aF/max(N,1) per order
            double aM = 0, aN = 0, aF = 0;
            for (int q = 0; q < P.nsym; ++q) {
                if (P.sym[q].unit != u || P.sym[q].slot != slot) continue;
                if (P.sym[q].kind == SYM_L_MEAN) aM += s_alpha[q];
                if (P.sym[q].kind == SYM_L_NSOLID) aN += s_alpha[q];
                if (P.sym[q].kind == SYM_L_FRAC) aF += s_alpha[q];
            }
            const double S1 = us[2 * slot], S0 = us[2 * slot + 1], N = us[4];
            const double W = fmax(S0, 1e-300);
            const double cv = S0 != 0.0 ? S1 / S0 : 0.0;
            U.coef[2 * slot] = aM / W;
            U.coef[2 * slot + 1] = -aM * cv / W + aN + aF / fmax(N, 1.0);
            if (slot == 0)
                for (int t = 4; t < 8; ++t) U.coef[t] = 0.0;
        } else if (slot == 0) {
            double c[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (U.kind == 0) {   // STEINH Q: c_ave = a/N, c_sw = a
                for (int q = 0; q < P.nsym; ++q) {
                    if (P.sym[q].unit != u) continue;
                    if (P.sym[q].kind == SYM_Q_AVE) c[0] += us[3] > 0 ? s_alpha[q] / us[3] : 0.0;
                    if (P.sym[q].kind == SYM_Q_SW) c[1 + P.sym[q].slot] += s_alpha[q];
                }
            } else if (U.kind == 2) {   // STRU_FACTOR: c_ave = a/N, c_count = a
                for (int q = 0; q < P.nsym; ++q) {
                    if (P.sym[q].unit != u) continue;
                    if (P.sym[q].kind == SYM_SF_AVE) c[0] += us[2] > 0 ? s_alpha[q] / us[2] : 0.0;
                    if (P.sym[q].kind == SYM_SF_COUNT) c[1] += s_alpha[q];
                }
            } else {   // S(k): 2 a / (N K)
                const double N = U.sk_n ? *U.sk_n : 0.0;
                for (int q = 0; q < P.nsym; ++q)
                    if (P.sym[q].unit == u && P.sym[q].kind == SYM_SK_AVE && N > 0 && U.K > 0)
                        c[0] += 2.0 * s_alpha[q] / (N * U.K);
            }
            for (int t = 0; t < 8; ++t) U.coef[t] = c[t];
        }
    }
}

struct BiasShared {
    double smem[8 * 32];
    double usum[kMaxUnits][8];
    double sv[kMaxDim];
    double sten[64];
    double s_sym[kMaxSymbols], s_jac[kMaxDim][kMaxSymbols], s_alpha[kMaxSymbols];
    double s_dV[kMaxDim], s_V;
    double row[3][16];
};

// One context, one step: all phases in one block.
__global__ void __launch_bounds__(256) k_bias_step(const BiasPlan *__restrict__ Pp, long long step) {
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ BiasShared S;
    // the plan is uploaded (and the stream synchronised) before a step's first
    // kernel, so it is staged while the CV kernel before this one drains
    stage_plan(Pp, plan_raw);
    pdl_entry();
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    phase_cvs(P, S.smem, S.usum, S.s_sym, S.s_jac, S.sv);
    const int dep = (P.pace != 0) && (step % P.pace == 0) && !step_failed(P);
    int ix[3] = {1, 1, 1};
    double fx[3] = {0, 0, 0};
    stencil_locate(P, S.sv, ix, fx);
    stencil_load(P, ix, S.sten);   // grid around s before this step's deposit
    __syncthreads();
    if (dep) {
        const double w = phase_wt_height(P, S.sten, fx, S.row, &S.s_V, S.s_dV);
        phase_deposit(P, S.sv, w, ix, S.sten);
        if (threadIdx.x == 0) record_hill(P, step, S.sv, w);
        __syncthreads();
    }
    phase_coef(P, S.sten, fx, S.sv, S.s_jac, S.usum, dep, S.row, &S.s_V, S.s_dV, S.s_alpha);
    if (P.save)
        for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) P.save->usum[e / 8][e % 8] = S.usum[e / 8][e % 8];
}

__global__ void __launch_bounds__(256) k_symbol_coef(const BiasPlan *__restrict__ Pp, int sym,
                                                     const WalkState *ws) {
    pdl_entry();
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ double usum[kMaxUnits][8], alpha[kMaxSymbols];
    stage_plan(Pp, plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) usum[e / 8][e % 8] = ws[0].usum[e / 8][e % 8];
    if (threadIdx.x < kMaxSymbols) alpha[threadIdx.x] = threadIdx.x == sym ? 1.0 : 0.0;
    __syncthreads();
    phase_unit_coefs(P, usum, alpha);
}

// ------------------------------------------------------------------ hill-list bias
__global__ void __launch_bounds__(256) k_list_cvs(const BiasPlan *__restrict__ Pp, WalkState *ws) {
    pdl_entry();
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ BiasShared S;
    stage_plan(Pp, plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    phase_cvs(P, S.smem, S.usum, S.s_sym, S.s_jac, S.sv);
    WalkState &W = ws[0];
    for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) W.usum[e / 8][e % 8] = S.usum[e / 8][e % 8];
    for (int e = threadIdx.x; e < kMaxDim * kMaxSymbols; e += blockDim.x)
        W.jac[e / kMaxSymbols][e % kMaxSymbols] = S.s_jac[e / kMaxSymbols][e % kMaxSymbols];
    if (threadIdx.x < kMaxDim) {
        const double v = threadIdx.x < P.D ? S.sv[threadIdx.x] : 0.0;
        W.s[threadIdx.x] = v;
        if (threadIdx.x < P.D) P.out[threadIdx.x] = v;   // read by the hill-sum / network kernels
    }
}

__global__ void __launch_bounds__(256) k_list_finish(const BiasPlan *__restrict__ Pp, long long step,
                                                     const WalkState *ws, const double *__restrict__ vdv) {
    pdl_entry();
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ BiasShared S;
    stage_plan(Pp, plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    const WalkState &W = ws[0];
    for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) S.usum[e / 8][e % 8] = W.usum[e / 8][e % 8];
    for (int e = threadIdx.x; e < kMaxDim * kMaxSymbols; e += blockDim.x)
        S.s_jac[e / kMaxSymbols][e % kMaxSymbols] = W.jac[e / kMaxSymbols][e % kMaxSymbols];
    const int dep = (P.pace != 0) && (step % P.pace == 0) && !step_failed(P);
    if (threadIdx.x < kMaxDim) {
        S.sv[threadIdx.x] = W.s[threadIdx.x];
        S.s_dV[threadIdx.x] = threadIdx.x < P.D ? vdv[1 + threadIdx.x] : 0.0;
    }
    if (threadIdx.x == 0) {
        double V = vdv[0];
        if (dep) {   // WT height from V(s) before the deposit (GH_t0_uniformGrid.cu:195-208)
            const double w = P.h0 * exp(-(P.wt ? V : 0.0) / (P.temp * P.kb * (P.biasf - 1.0)));
            record_hill(P, step, W.s, w);
            V += w;
        }
        S.s_V = V;
    }
    __syncthreads();
    phase_coef_from_v(P, S.sv, S.s_jac, S.usum, dep, &S.s_V, S.s_dV, S.s_alpha);
}

// ------------------------------------------------------------------ multiple walkers
// W walkers share one grid.  A: per walker (one block each) the CV values and,
// on a deposit step, the WT height from the grid as it stands at the start of
// the step.  B: the W hills deposited in walker order (one block; every bin
// receives its increments in walker order).  C: per walker V, dV/ds on the
// updated grid and the force coefficients.  The step is read from device
// memory so the three launches can sit in a CUDA graph.
// Walker w's CVs (one block): totals, symbols, DIM values, and on a deposit
// step the WT height from the grid as it stood at the start of the step.
__device__ void walk_cvs_block(const BiasPlan *const *__restrict__ plans, int w, const long long *__restrict__ d_step,
                               WalkState *ws) {
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ BiasShared S;
    stage_plan(plans[w], plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    const long long step = *(volatile const long long *)d_step;
    phase_cvs(P, S.smem, S.usum, S.s_sym, S.s_jac, S.sv);
    const int dep = (P.pace != 0) && (step % P.pace == 0) && !step_failed(P);
    WalkState &W = ws[w];
    if (dep) {
        int ix[3] = {1, 1, 1};
        double fx[3] = {0, 0, 0};
        stencil_locate(P, S.sv, ix, fx);
        stencil_load(P, ix, S.sten);
        __syncthreads();
        const double w = phase_wt_height(P, S.sten, fx, S.row, &S.s_V, S.s_dV);
        if (threadIdx.x == 0) W.hill_w = w;
    }
    for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) W.usum[e / 8][e % 8] = S.usum[e / 8][e % 8];
    for (int e = threadIdx.x; e < kMaxDim * kMaxSymbols; e += blockDim.x)
        W.jac[e / kMaxSymbols][e % kMaxSymbols] = S.s_jac[e / kMaxSymbols][e % kMaxSymbols];
    if (threadIdx.x < kMaxDim) W.s[threadIdx.x] = threadIdx.x < P.D ? S.sv[threadIdx.x] : 0.0;
    if (threadIdx.x == 0) W.dep = dep;
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_walk_cvs(const BiasPlan *const *__restrict__ plans,
                                                  const long long *__restrict__ d_step, WalkState *ws) {
    pdl_entry();
    walk_cvs_block(plans, blockIdx.x, d_step, ws);
}

// True (in every thread) when any walker's neighbour lists overflowed this
// step: the host repeats the whole group's step, so no walker may deposit or
// apply a bias force.
__device__ bool group_failed(const BiasPlan *const *__restrict__ plans, int nwalk) {
    __shared__ int failed;
    if (threadIdx.x == 0) failed = 0;
    __syncthreads();
    for (int w = threadIdx.x; w < nwalk; w += blockDim.x) {
        const DevStatus *st = plans[w]->status;
        if (status_failed(st)) failed = 1;
    }
    __syncthreads();
    return failed != 0;
}

// The group's hills in walker order, spread over every thread of the
// launch (vblock / nvblocks: this block's place among the blocks taking
// part): each bin of the bands' bounding box takes, in walker order, the
// increment of every walker whose band holds it -- per bin the same
// operations as depositing the hills one after another, so the grid is the
// same bit for bit.  Block 0's first thread writes the hill records in
// walker order.
__device__ void walk_deposit_block(const BiasPlan *const *__restrict__ plans, int nwalk,
                                   const long long *__restrict__ d_step, const WalkState *ws, int vblock,
                                   int nvblocks) {
    const BiasPlan &P = *plans[0];
    const bool failed = group_failed(plans, nwalk);
    const long long step = *(volatile const long long *)d_step;
    if (failed || P.pace == 0 || step % P.pace != 0) return;   // every walker shares PACE
    __shared__ int bb[6];
    if (threadIdx.x < 3) {
        bb[threadIdx.x] = 0x7fffffff;
        bb[3 + threadIdx.x] = -1;
    }
    __syncthreads();
    for (int w = threadIdx.x; w < nwalk; w += blockDim.x) {
        int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        if (!hill_band(P, ws[w].s, lo, hi)) continue;
        for (int k = 0; k < P.D; ++k) {
            atomicMin(&bb[k], lo[k]);
            atomicMax(&bb[3 + k], hi[k]);
        }
    }
    __syncthreads();
    if (vblock == 0 && threadIdx.x == 0)
        for (int w = 0; w < nwalk; ++w) record_hill(P, step, ws[w].s, ws[w].hill_w);
    long long total = 1;
    int ext[3] = {1, 1, 1};
    for (int k = 0; k < P.D; ++k) {
        ext[k] = bb[3 + k] - bb[k] + 1;
        total = ext[k] > 0 ? total * ext[k] : 0;
    }
    for (long long t = (long long)vblock * blockDim.x + threadIdx.x; t < total; t += (long long)nvblocks * blockDim.x) {
        int idx[3] = {0, 0, 0};
        long long rem = t;
        for (int k = P.D - 1; k >= 0; --k) {
            idx[k] = bb[k] + (int)(rem % ext[k]);
            rem /= ext[k];
        }
        size_t g = idx[0];
        for (int k = 1; k < P.D; ++k) g = g * P.nbin[k] + idx[k];
        if (g >= (size_t)P.grid_size) continue;
        double v = 0.0;
        bool any = false;
        for (int w = 0; w < nwalk; ++w) {
            int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            if (!hill_band(P, ws[w].s, lo, hi)) continue;
            bool in = true;
            for (int k = 0; k < P.D; ++k) in = in && idx[k] >= lo[k] && idx[k] <= hi[k];
            if (!in) continue;
            if (!any) v = __ldcg(P.grid + g);
            any = true;
            v = v + ws[w].hill_w * hill_gauss(P, ws[w].s, idx, P.sigma);
        }
        if (any) P.grid[g] = v;
    }
}

__global__ void __launch_bounds__(256) k_walk_deposit(const BiasPlan *const *__restrict__ plans, int nwalk,
                                                      const long long *__restrict__ d_step, const WalkState *ws) {
    pdl_entry();
    walk_deposit_block(plans, nwalk, d_step, ws, blockIdx.x, gridDim.x);
}

// Walker w's V, dV/ds on the updated grid and force coefficients (one block).
__device__ void walk_coef_block(const BiasPlan *const *__restrict__ plans, int nwalk, int w, const WalkState *ws) {
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ BiasShared S;
    stage_plan(plans[w], plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    if (group_failed(plans, nwalk)) {
        for (int e = threadIdx.x; e < P.nunit * 8; e += blockDim.x) P.unit[e / 8].coef[e % 8] = 0.0;
        __syncthreads();
        return;
    }
    const WalkState &W = ws[w];
    for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) S.usum[e / 8][e % 8] = W.usum[e / 8][e % 8];
    for (int e = threadIdx.x; e < kMaxDim * kMaxSymbols; e += blockDim.x)
        S.s_jac[e / kMaxSymbols][e % kMaxSymbols] = W.jac[e / kMaxSymbols][e % kMaxSymbols];
    if (threadIdx.x < kMaxDim) S.sv[threadIdx.x] = W.s[threadIdx.x];
    __syncthreads();
    int ix[3] = {1, 1, 1};
    double fx[3] = {0, 0, 0};
    stencil_locate(P, S.sv, ix, fx);
    stencil_load(P, ix, S.sten);
    __syncthreads();
    phase_coef(P, S.sten, fx, S.sv, S.s_jac, S.usum, W.dep, S.row, &S.s_V, S.s_dV, S.s_alpha);
    __syncthreads();
}

__global__ void __launch_bounds__(256) k_walk_coef(const BiasPlan *const *__restrict__ plans, int nwalk,
                                                   const WalkState *ws) {
    pdl_entry();
    walk_coef_block(plans, nwalk, blockIdx.x, ws);
}

// ---- walkers sharded over ranks: each rank steps its own walkers; their
// hills are exchanged (kWalkRec doubles per walker: s[kMaxDim], height,
// deposit flag, neighbour-overflow flag, 0) and every rank deposits all
// ranks' hills in global walker order, so every grid stays the same.
__global__ void k_walk_pack(const BiasPlan *const *__restrict__ plans, int nwalk, const WalkState *ws, double *out) {
    pdl_entry();
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nwalk) return;
    double *r = out + (size_t)k * kWalkRec;
    for (int d = 0; d < kMaxDim; ++d) r[d] = ws[k].s[d];
    r[kMaxDim] = ws[k].hill_w;
    r[kMaxDim + 1] = ws[k].dep ? 1.0 : 0.0;
    const DevStatus *st = plans[k]->status;
    r[kMaxDim + 2] = status_failed(st) ? 1.0 : 0.0;
    r[kMaxDim + 3] = 0.0;
}

// Any walker of any rank overflowed its neighbour lists this step.
__device__ bool all_failed(const double *__restrict__ recs, int nrec) {
    __shared__ int failed;
    if (threadIdx.x == 0) failed = 0;
    __syncthreads();
    for (int r = threadIdx.x; r < nrec; r += blockDim.x)
        if (recs[(size_t)r * kWalkRec + kMaxDim + 2] != 0.0) failed = 1;
    __syncthreads();
    return failed != 0;
}

__global__ void __launch_bounds__(256) k_walk_deposit_all(const BiasPlan *const *__restrict__ plans,
                                                          const long long *__restrict__ d_step,
                                                          const double *__restrict__ recs, int nrec) {
    pdl_entry();
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    stage_plan(plans[0], plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    if (all_failed(recs, nrec)) return;
    const long long step = *d_step;
    if (!(P.pace != 0 && step % P.pace == 0)) return;   // every walker shares PACE
    int ix[3] = {1, 1, 1};
    for (int r = 0; r < nrec; ++r) {
        const double *rec = recs + (size_t)r * kWalkRec;
        phase_deposit(P, rec, rec[kMaxDim], ix, nullptr);
        if (threadIdx.x == 0) record_hill(P, step, rec, rec[kMaxDim]);
        __syncthreads();
    }
}

__global__ void __launch_bounds__(256) k_walk_coef_all(const BiasPlan *const *__restrict__ plans, const WalkState *ws,
                                                       const double *__restrict__ recs, int nrec) {
    pdl_entry();
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ BiasShared S;
    stage_plan(plans[blockIdx.x], plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    if (all_failed(recs, nrec)) {
        for (int e = threadIdx.x; e < P.nunit * 8; e += blockDim.x) P.unit[e / 8].coef[e % 8] = 0.0;
        return;
    }
    const WalkState &W = ws[blockIdx.x];
    for (int e = threadIdx.x; e < kMaxUnits * 8; e += blockDim.x) S.usum[e / 8][e % 8] = W.usum[e / 8][e % 8];
    for (int e = threadIdx.x; e < kMaxDim * kMaxSymbols; e += blockDim.x)
        S.s_jac[e / kMaxSymbols][e % kMaxSymbols] = W.jac[e / kMaxSymbols][e % kMaxSymbols];
    if (threadIdx.x < kMaxDim) S.sv[threadIdx.x] = W.s[threadIdx.x];
    __syncthreads();
    int ix[3] = {1, 1, 1};
    double fx[3] = {0, 0, 0};
    stencil_locate(P, S.sv, ix, fx);
    stencil_load(P, ix, S.sten);
    __syncthreads();
    phase_coef(P, S.sten, fx, S.sv, S.s_jac, S.usum, W.dep, S.row, &S.s_V, S.s_dV, S.s_alpha);
}

// HILLS replay: every thread owns grid bins and adds the hills in file order,
// so the FP64 sum order per bin is the file order.
__global__ void k_hills_replay(const BiasPlan *__restrict__ Pp, const HillRec *__restrict__ h, int nh, int ncell) {
    pdl_entry();
    const BiasPlan &P = *Pp;
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < ncell; g += gridDim.x * blockDim.x) {
        int idx[3] = {0, 0, 0}, rem = g;
        for (int k = P.D - 1; k >= 0; --k) {
            idx[k] = rem % P.nbin[k];
            rem /= P.nbin[k];
        }
        double acc = P.grid[g];
        for (int q = 0; q < nh; ++q) {
            int lo[3], hi[3];
            if (!hill_band(P, h[q].s, lo, hi)) continue;
            bool in = true;
            for (int k = 0; k < P.D; ++k) in = in && idx[k] >= lo[k] && idx[k] <= hi[k];
            if (in) acc += h[q].w * hill_gauss(P, h[q].s, idx, h[q].sigma);
        }
        P.grid[g] = acc;
    }
}

__global__ void k_virial_finalize(const double *__restrict__ vpart, int nparts, double *out6) {
    pdl_entry();
    __shared__ double smem[6 * 32];
    double v[6] = {0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nparts; b += blockDim.x)
        for (int t = 0; t < 6; ++t) v[t] += vpart[(size_t)b * 8 + t];
    block_sum<6>(v, smem);
    if (threadIdx.x == 0)
        for (int t = 0; t < 6; ++t) out6[t] = v[t];
}

}  // namespace

// The three bias phases of the multi-walker step as block-level functions
// for the persistent step kernel (walk_step.cu), compiled here with this
// file's arithmetic.
__device__ void walk_phase_cvs(const BiasPlan *const *plans, int w, const long long *d_step, WalkState *ws) {
    walk_cvs_block(plans, w, d_step, ws);
}
__device__ void walk_phase_deposit(const BiasPlan *const *plans, int nwalk, const long long *d_step,
                                   const WalkState *ws, int vblock, int nvblocks) {
    walk_deposit_block(plans, nwalk, d_step, ws, vblock, nvblocks);
}
__device__ void walk_phase_coef(const BiasPlan *const *plans, int nwalk, int w, const WalkState *ws) {
    walk_coef_block(plans, nwalk, w, ws);
}

__global__ void __launch_bounds__(256) k_unit_sums(const BiasPlan *__restrict__ Pp, double *out) {
    pdl_entry();
    __shared__ __align__(16) unsigned char plan_raw[sizeof(BiasPlan)];
    __shared__ double smem[8 * 32];
    stage_plan(Pp, plan_raw);
    const BiasPlan &P = *reinterpret_cast<const BiasPlan *>(plan_raw);
    for (int u = 0; u < P.nunit; ++u) unit_total(P.unit[u], smem, out + 8 * u);
    int off = 8 * P.nunit;
    for (int u = 0; u < P.nunit; ++u) {
        const UnitPlan &U = P.unit[u];
        if (!U.rho) continue;
        for (int t = threadIdx.x; t < 2 * U.K; t += blockDim.x) out[off + t] = U.rho[t];
        if (threadIdx.x == 0) out[off + 2 * U.K] = *U.sk_n;
        off += 2 * U.K + 1;
    }
    if (threadIdx.x == 0) {
        out[off] = P.status ? (double)max(P.status->overflow, P.status->cand_overflow) : 0.0;
        out[off + 1] = P.status ? (double)P.status->bad_pos : 0.0;
    }
}

int unit_sums_count(const BiasPlan &P) {
    int c = 8 * P.nunit + 2;   // + the neighbour-overflow and non-finite-position flags
    for (int u = 0; u < P.nunit; ++u)
        if (P.unit[u].rho) c += 2 * P.unit[u].K + 1;
    return c;
}

void launch_unit_sums(const BiasPlan *d_plan, double *out, cudaStream_t st) {
    launch_k(k_unit_sums, 1, 256, 0, st, d_plan, out);
    prof_mark("unit_sums", st);
}

// Domain decomposition with a device-side allreduce: the summed overflow
// counts of all ranks mark this rank's step failed too (flag 1: nothing to
// grow), and so does a non-finite position on any rank (no rank deposits,
// every rank reports it).  gflag[0]: overflow sum, gflag[1]: bad-position sum.
__global__ void k_domain_flag(const double *gflag, DevStatus *status) {
    pdl_entry();
    if (threadIdx.x == 0) {
        if (gflag[0] != 0.0 && status->overflow == 0u) status->overflow = 1u;
        if (gflag[1] != 0.0) status->bad_pos = 1u;
    }
}

void launch_domain_flag(const double *gflag, DevStatus *status, cudaStream_t st) {
    launch_k(k_domain_flag, 1, 32, 0, st, gflag, status);
}

void launch_bias_step(const BiasPlan *d_plan, long long step, cudaStream_t st) {
    launch_k(k_bias_step, 1, 256, 0, st, d_plan, step);
    prof_mark("bias_step", st);
}

void launch_symbol_coef(const BiasPlan *d_plan, int sym, const WalkState *ws, cudaStream_t st) {
    launch_k(k_symbol_coef, 1, 256, 0, st, d_plan, sym, ws);
}

void launch_list_cvs(const BiasPlan *d_plan, WalkState *ws, cudaStream_t st) {
    launch_k(k_list_cvs, 1, 256, 0, st, d_plan, ws);
    prof_mark("bias_cvs", st);
}

void launch_list_finish(const BiasPlan *d_plan, long long step, const WalkState *ws, const double *vdv,
                        cudaStream_t st) {
    launch_k(k_list_finish, 1, 256, 0, st, d_plan, step, ws, vdv);
    prof_mark("bias_finish", st);
}

void launch_walk_bias(const BiasPlan *const *d_plans, int nwalk, const long long *d_step, WalkState *ws,
                      cudaStream_t st) {
    launch_k(k_walk_cvs, nwalk, 256, 0, st, d_plans, d_step, ws);
    launch_k(k_walk_deposit, 148, 256, 0, st, d_plans, nwalk, d_step, ws);
    launch_k(k_walk_coef, nwalk, 256, 0, st, d_plans, nwalk, ws);
    prof_mark("walk_bias", st);
}

void launch_walk_cvs_pack(const BiasPlan *const *d_plans, int nwalk, const long long *d_step, WalkState *ws,
                          double *out, cudaStream_t st) {
    launch_k(k_walk_cvs, nwalk, 256, 0, st, d_plans, d_step, ws);
    launch_k(k_walk_pack, (nwalk + 127) / 128, 128, 0, st, d_plans, nwalk, (const WalkState *)ws, out);
}

void launch_walk_finish(const BiasPlan *const *d_plans, int nwalk, const long long *d_step, const WalkState *ws,
                        const double *recs, int nrec, cudaStream_t st) {
    launch_k(k_walk_deposit_all, 1, 256, 0, st, d_plans, d_step, recs, nrec);
    launch_k(k_walk_coef_all, nwalk, 256, 0, st, d_plans, ws, recs, nrec);
    prof_mark("walk_bias", st);
}

void launch_hills_replay(const BiasPlan *d_plan, const HillRec *h, int nh, int ncell, cudaStream_t st) {
    if (nh <= 0 || ncell <= 0) return;
    int blocks = (ncell + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    launch_k(k_hills_replay, blocks, 256, 0, st, d_plan, h, nh, ncell);
}

void launch_virial_finalize(const double *vpart, int nparts, double *out6, cudaStream_t st) {
    launch_k(k_virial_finalize, 1, 256, 0, st, vpart, nparts, out6);
    prof_mark("virial", st);
}

}  // namespace mtd
