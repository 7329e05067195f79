// local_ql.cu -- STEINH L (local-averaged Q_l) values and analytic forces.
//
// Replaces steinhardt_Local_cv_get_qlm / _get_LQl
// (src/cvs/CVs_Steinhardt_Local.cu:1309-1580), the MEAN_SOLID / NSOLID / FRAC
// reductions (:695-745, src/utils/CVs_tools.cu:20-55) and the ij + jk force
// kernels with FP64 atomics (:1622-2130).
//
// Definitions (sigma = SW_FUNC_r, N(i) = {j : sigma(r_ij) >= eps}):
//   NF_i = sum_j sigma_ij,  q_i = sum_j sigma_ij Y(d_ij) / NF_i,
//   LQ_i = (q_i + sum_j sigma_ij q_j) / (NF_i + 1),  LQ_i = |LQ_i|_l.
// Forces use an adjoint (gather) formulation with no atomics, so FP64 runs are
// bitwise reproducible.  For each atom
//   G_i   = dCV/dLQ_i * (4 pi/(2l+1)) / LQ_i * w_m LQ_lm,i / (NF_i + 1)
//   lam_k = G_k + sum_{i in N(k)} sigma_ki G_i                  (adjoint of q_k)
// and the gradient on atom a gathers over its neighbours j with
//   Lam = lam_a/NF_a + (-1)^l lam_j/NF_j,
//   dCV/dx_a = - sum_j [ sigma grad_d Re(Lam . Y(d_aj))
//                        + sigma' dhat (c_aj + c_ja + Re(Lam . Y) - t_a - t_j) ]
// where c_aj = Re G_a.(q_j - LQ_a), t_a = Re lam_a.q_a / NF_a.  Two orders
// (Q4 and Q6 of one neighbour environment) are fused in one pass.  With a STEP
// switch sigma = 1 and sigma' = 0 on every listed pair, so the LQ and lambda
// passes need neighbour indices only.
#include "local_body.cuh"

namespace mtd {

namespace {

// The passes as kernels (local_body.cuh).
template <int LA, int LB, typename T, bool STEP, bool FILTER, bool MERGED = true>
__global__ void __launch_bounds__(kBlock, 4) k_local_q(LocalDev<T> d) {
    pdl_entry();
    local_q_body<LA, LB, T, STEP, FILTER, MERGED>(d, blockIdx.x);
}

template <int LA, int LB, typename T, bool STEP>
__global__ void __launch_bounds__(kBlock, 4) k_local_lq(LocalDev<T> d) {
    pdl_entry();
    local_lq_body<LA, LB, T, STEP>(d, blockIdx.x);
}

template <int LA, int LB, typename T, bool STEP>
__global__ void __launch_bounds__(kBlock) k_local_lambda(LocalDev<T> d) {
    local_lambda_body<LA, LB, T, STEP>(d, blockIdx.x, true);   // the body places the wait
}

template <int LA, int LB, typename T, bool STEP, bool CALLER = false>
__global__ void __launch_bounds__(kBlock, CALLER ? 2 : 4) k_local_force(LocalDev<T> d, const double *__restrict__ f_src,
                                                        double *__restrict__ f_dst, SysDev s, CellGrid g,
                                                        double *vpart, DevStatus *status) {
    pdl_entry();
    local_force_body<LA, LB, T, STEP, CALLER>(d, f_src, f_dst, s, g, vpart, status, blockIdx.x);
}

template <int LA, int LB, typename T> void run_values(const LocalDev<T> &d, cudaStream_t st) {
    const int nb = (d.n + kBlock - 1) / kBlock;
    const int qb = d.qblock > 0 ? d.qblock : kBlock, qg = (d.n + qb - 1) / qb;   // no block reduction in q
    if (d.sw_r.type == SW_STEP) {
        if (d.filter && d.qsplit) launch_k(k_local_q<LA, LB, T, true, true, false>, qg, qb, 0, st, d);
        else if (d.filter) launch_k(k_local_q<LA, LB, T, true, true>, qg, qb, 0, st, d);
        else launch_k(k_local_q<LA, LB, T, true, false>, qg, qb, 0, st, d);
        prof_mark("local_q", st);
        launch_k(k_local_lq<LA, LB, T, true>, nb, kBlock, 0, st, d);
        prof_mark("local_lq", st);
    } else {
        if (d.filter && d.qsplit) launch_k(k_local_q<LA, LB, T, false, true, false>, qg, qb, 0, st, d);
        else if (d.filter) launch_k(k_local_q<LA, LB, T, false, true>, qg, qb, 0, st, d);
        else launch_k(k_local_q<LA, LB, T, false, false>, qg, qb, 0, st, d);
        prof_mark("local_q", st);
        launch_k(k_local_lq<LA, LB, T, false>, nb, kBlock, 0, st, d);
        prof_mark("local_lq", st);
    }
}

template <int LA, int LB, typename T> void run_lambda(const LocalDev<T> &d, cudaStream_t st) {
    const int lb = d.lblock > 0 ? d.lblock : kBlock, lg = (d.n + lb - 1) / lb;
    if (d.sw_r.type == SW_STEP) launch_k(k_local_lambda<LA, LB, T, true>, lg, lb, 0, st, d);
    else launch_k(k_local_lambda<LA, LB, T, false>, lg, lb, 0, st, d);
    prof_mark("local_lambda", st);
}

template <int LA, int LB, typename T>
void run_force_pass(const LocalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                    double *vpart, DevStatus *status, cudaStream_t st) {
    const int cnt = d.iperm ? d.i1 - d.i0 : d.n;
    if (cnt <= 0) return;
    const int nb = (cnt + kBlock - 1) / kBlock;
    if (d.iperm) {
        if (d.sw_r.type == SW_STEP)
            launch_k(k_local_force<LA, LB, T, true, true>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
        else
            launch_k(k_local_force<LA, LB, T, false, true>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
    } else if (d.sw_r.type == SW_STEP) {
        launch_k(k_local_force<LA, LB, T, true>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
    } else {
        launch_k(k_local_force<LA, LB, T, false>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
    }
    prof_mark("local_force", st);
}

template <int LA, int LB, typename T>
void run_forces(const LocalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                double *vpart, DevStatus *status, cudaStream_t st) {
    const int nb = (d.n + kBlock - 1) / kBlock;
    const int lb = d.lblock > 0 ? d.lblock : kBlock, lg = (d.n + lb - 1) / lb;   // no block reduction in lambda
    if (d.sw_r.type == SW_STEP) {
        launch_k(k_local_lambda<LA, LB, T, true>, lg, lb, 0, st, d);
        prof_mark("local_lambda", st);
        launch_k(k_local_force<LA, LB, T, true>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
        prof_mark("local_force", st);
    } else {
        launch_k(k_local_lambda<LA, LB, T, false>, lg, lb, 0, st, d);
        prof_mark("local_lambda", st);
        launch_k(k_local_force<LA, LB, T, false>, nb, kBlock, 0, st, d, f_src, f_dst, s, g, vpart, status);
        prof_mark("local_force", st);
    }
}

}  // namespace

#define MTD_LOCAL_DISPATCH(FN, ...)                                                          \
    do {                                                                                     \
        const int key = d.LA * 16 + d.LB;                                                    \
        switch (key) {                                                                       \
        case 3 * 16: FN<3, 0, T>(__VA_ARGS__); break;                                        \
        case 4 * 16: FN<4, 0, T>(__VA_ARGS__); break;                                        \
        case 6 * 16: FN<6, 0, T>(__VA_ARGS__); break;                                        \
        case 4 * 16 + 6: FN<4, 6, T>(__VA_ARGS__); break;                                    \
        case 6 * 16 + 4: FN<6, 4, T>(__VA_ARGS__); break;                                    \
        case 3 * 16 + 4: FN<3, 4, T>(__VA_ARGS__); break;                                    \
        case 3 * 16 + 6: FN<3, 6, T>(__VA_ARGS__); break;                                    \
        default: break;                                                                      \
        }                                                                                    \
    } while (0)

int local_record_stride(int LA, int LB, int fp64) {
    const int n = 2 * (LA + 1) + (LB ? 2 * (LB + 1) : 0);
    const int v = fp64 ? 4 : 8;
    return (n + v - 1) / v * v;
}

template <typename T> void launch_local_values(const LocalDev<T> &d, cudaStream_t st) {
    if (d.n == 0) return;
    MTD_LOCAL_DISPATCH(run_values, d, st);
}

template <typename T>
void launch_local_forces(const LocalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                         double *vpart, DevStatus *status, cudaStream_t st) {
    if (d.n == 0) return;
    MTD_LOCAL_DISPATCH(run_forces, d, f_src, f_dst, s, g, vpart, status, st);
}

template <typename T> void launch_local_lambda(const LocalDev<T> &d, cudaStream_t st) {
    if (d.n == 0) return;
    MTD_LOCAL_DISPATCH(run_lambda, d, st);
}

template <typename T>
void launch_local_force_pass(const LocalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s,
                             const CellGrid &g, double *vpart, DevStatus *status, cudaStream_t st) {
    if (d.n == 0) return;
    MTD_LOCAL_DISPATCH(run_force_pass, d, f_src, f_dst, s, g, vpart, status, st);
}

template void launch_local_lambda<float>(const LocalDev<float> &, cudaStream_t);
template void launch_local_lambda<double>(const LocalDev<double> &, cudaStream_t);
template void launch_local_force_pass<float>(const LocalDev<float> &, const double *, double *, const SysDev &,
                                             const CellGrid &, double *, DevStatus *, cudaStream_t);
template void launch_local_force_pass<double>(const LocalDev<double> &, const double *, double *, const SysDev &,
                                              const CellGrid &, double *, DevStatus *, cudaStream_t);
template void launch_local_values<float>(const LocalDev<float> &, cudaStream_t);
template void launch_local_values<double>(const LocalDev<double> &, cudaStream_t);
template void launch_local_forces<float>(const LocalDev<float> &, const double *, double *, const SysDev &,
                                         const CellGrid &, double *, DevStatus *, cudaStream_t);
template void launch_local_forces<double>(const LocalDev<double> &, const double *, double *, const SysDev &,
                                          const CellGrid &, double *, DevStatus *, cudaStream_t);

}  // namespace mtd
