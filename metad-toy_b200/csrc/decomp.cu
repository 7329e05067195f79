// decomp.cu -- domain decomposition across ranks (one context per rank): the
// per-step exchange of every unit's totals through the caller's allreduce,
// and the C-ABI calls that set it up.  The reference's CVs reduce their local
// sums with MPI_Allreduce under LAMMPS's decomposition
// (src/cvs/CVs_Steinhardt.cu:836, src/cvs/CVs_Strufactor.cu:653, :671).
#include "context.h"

namespace mtd {
namespace ctx {

// Domain decomposition, between the CV passes and the bias kernel: this
// rank's unit totals (and S(k) sums, its neighbour-overflow flag and its
// non-finite-position flag) go to the caller's allreduce; the totals over all
// ranks come back for the bias kernel (P.gsum) and the S(k) arrays.  A step
// that overflowed on any rank counts as overflowed on every rank, so all
// ranks skip the deposit and, in mtd_post_force, retry together; a
// non-finite position on any rank makes every rank skip the deposit and the
// bias force and return MTD_ERR_NAN.
mtd_status exchange_totals(mtd_ctx *c) {
    const int cnt = c->xchg_n;
    launch_unit_sums(c->d_plan, c->d_xchg, c->st);
    c->launches += 1;
    if (c->dom_dev_fn) {   // the caller enqueues the sum over ranks on the step's stream
        if (c->dom_dev_fn(c->d_xchg, cnt, (void *)c->st, c->dom_user) != 0)
            return fail(c, MTD_ERR_INVALID_ARG, "domain decomposition: the device allreduce callback failed");
        MTD_CU(cudaGetLastError(), "domain allreduce");
        int off = 8 * (int)c->units.size();
        for (Unit &u : c->units) {
            if (u.kind != CAL_STRU_FACTOR_K) continue;
            MTD_CU(cudaMemcpyAsync(u.rho, c->d_xchg + off, sizeof(double) * 2 * u.K, cudaMemcpyDeviceToDevice, c->st), "rho(k)");
            MTD_CU(cudaMemcpyAsync(u.skn, c->d_xchg + off + 2 * u.K, sizeof(double), cudaMemcpyDeviceToDevice, c->st), "rho(k)");
            off += 2 * u.K + 1;
        }
        launch_domain_flag(c->d_xchg + cnt - 2, c->d_status, c->st);   // any rank overflowed: every rank retries
        c->launches += 1;
        return MTD_OK;
    }
    MTD_CU(cudaMemcpyAsync(c->h_xchg, c->d_xchg, sizeof(double) * cnt, cudaMemcpyDeviceToHost, c->st), "domain totals");
    MTD_CU(cudaStreamSynchronize(c->st), "domain totals");
    const double own_overflow = c->h_xchg[cnt - 2];
    if (c->dom_fn(c->h_xchg, cnt, c->dom_user) != 0)
        return fail(c, MTD_ERR_INVALID_ARG, "domain decomposition: the allreduce callback failed");
    MTD_CU(cudaMemcpyAsync(c->d_xchg, c->h_xchg, sizeof(double) * cnt, cudaMemcpyHostToDevice, c->st), "domain totals");
    int off = 8 * (int)c->units.size();
    for (Unit &u : c->units) {
        if (u.kind != CAL_STRU_FACTOR_K) continue;
        MTD_CU(cudaMemcpyAsync(u.rho, c->d_xchg + off, sizeof(double) * 2 * u.K, cudaMemcpyDeviceToDevice, c->st), "rho(k)");
        MTD_CU(cudaMemcpyAsync(u.skn, c->d_xchg + off + 2 * u.K, sizeof(double), cudaMemcpyDeviceToDevice, c->st), "rho(k)");
        off += 2 * u.K + 1;
    }
    if (c->h_xchg[cnt - 2] != 0.0 && own_overflow == 0.0)   // another rank overflowed: a flag of 1 (no growth here)
        MTD_CU(cudaMemsetAsync(&c->d_status->overflow, 1, 1, c->st), "status");
    if (c->h_xchg[cnt - 1] != 0.0)   // a non-finite position on any rank: no rank deposits, every rank reports it
        MTD_CU(cudaMemsetAsync(&c->d_status->bad_pos, 1, 1, c->st), "status");
    return MTD_OK;
}

}  // namespace ctx
}  // namespace mtd

extern "C" {

mtd_status mtd_set_domain(mtd_ctx *c, int nlocal, int rank, mtd_allreduce_fn fn, void *user) {
    if (!c) return MTD_ERR_INVALID_ARG;
    if (c->initialized)
        return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_domain must be called before the first step");
    if (nlocal < 0 || rank < 0 || !fn)
        return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_domain needs nlocal >= 0, rank >= 0 and an allreduce callback");
    if (c->cfg.hill_list())
        return fail(c, MTD_ERR_UNSUPPORTED, "domain decomposition needs the grid bias (CV_dim 1-3, no NN_BIAS)");
    c->nown = nlocal;
    c->dom_rank = rank;
    c->dom_fn = fn;
    c->dom_user = user;
    c->plan_dirty = true;
    return MTD_OK;
}

mtd_status mtd_set_domain_device(mtd_ctx *c, int nlocal, int rank, mtd_allreduce_device_fn fn, void *user) {
    if (!c || !fn) return MTD_ERR_INVALID_ARG;
    const mtd_status s = mtd_set_domain(c, nlocal, rank, reinterpret_cast<mtd_allreduce_fn>(fn), user);
    if (s != MTD_OK) return s;
    c->dom_fn = nullptr;
    c->dom_dev_fn = fn;
    return MTD_OK;
}

mtd_status mtd_set_nlocal(mtd_ctx *c, int nlocal) {
    if (!c || nlocal < 0) return MTD_ERR_INVALID_ARG;
    if (c->nown < 0) return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_nlocal: domain decomposition is not enabled");
    c->nown = nlocal;
    return MTD_OK;
}

double mtd_ghost_cutoff(const mtd_ctx *c) {
    if (!c) return 0.0;
    double g = 0.0;
    for (const Env &e : c->envs) g = std::fmax(g, e.kind == ENV_L ? 2.0 * e.rc : e.rc);
    // skin lists: atoms move up to skin / 2 between rebuilds, so the shell
    // taken at a rebuild must reach that much further for each of the two
    if (g > 0.0 && c->cfg.neigh_skin > 0.0) g += c->cfg.neigh_skin;
    return g;
}

}  // extern "C"
