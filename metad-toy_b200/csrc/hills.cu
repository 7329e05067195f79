// hills.cu -- the HILLS file (rows written as hills are collected, restart
// replay into the grid) and the hill-list bias bookkeeping (new hills join
// the exact sum; periodic refits of the learned bias).
// HILLS format and restart: src/grids/GH_t0_uniformGrid.cu:101-220.
#include "context.h"

namespace mtd {
namespace ctx {

void write_hill_line(mtd_ctx *c, const HillRec &h) {
    if (!c->f_hills) return;
    std::fprintf(c->f_hills, "%lld", h.step);   // GH_t0_uniformGrid.cu:211-220
    for (int d = 0; d < c->cfg.cv_dim; ++d) std::fprintf(c->f_hills, " %.16g", h.s[d]);
    std::fprintf(c->f_hills, " %.16g %.16g\n", h.w, h.sigma);
    std::fflush(c->f_hills);
}

// Hill-list bias: new hills join the exact sum; every NN_REFIT hills the
// network is refitted on the sum and validated against it (the exact sum, plus
// the network when it passes, is what the next steps use).
mtd_status list_add_hills(mtd_ctx *c, const std::vector<HillRec> &recs) {
    const int D = c->cfg.cv_dim;
    std::vector<double> cen, hgt, sig;
    for (const HillRec &r : recs) {
        for (int d = 0; d < D; ++d) cen.push_back(r.s[d]);
        hgt.push_back(r.w);
        sig.push_back(r.sigma);
    }
    if (!hgt.empty() && mtd_nnbias_add_hills(c->nb, (int)hgt.size(), cen.data(), hgt.data(), sig.data()) != MTD_OK)
        return fail(c, MTD_ERR_CUDA, mtd_nnbias_last_error(c->nb));
    const int nh = mtd_nnbias_num_hills(c->nb);
    if (c->cfg.nn && nh - c->h_fit >= c->cfg.nn_refit) {
        double loss = 0.0, mx = 0.0, rms = 0.0;
        if (mtd_nnbias_fit(c->nb, 65536, c->cfg.nn_iters, 4096, 2e-3, 1000 + (unsigned long long)nh, &loss) != MTD_OK ||
            mtd_nnbias_validate(c->nb, 16384, 7 + (unsigned long long)nh, c->cfg.nn_tol, &mx, &rms) != MTD_OK)
            return fail(c, MTD_ERR_CUDA, mtd_nnbias_last_error(c->nb));
        c->h_fit = nh;
        c->nn_usable = mtd_nnbias_usable(c->nb) != 0;
    }
    return MTD_OK;
}

std::string path_in(const mtd_ctx *c, const std::string &p) {
    if (p.empty() || p[0] == '/' || c->work_dir.empty()) return p;
    return c->work_dir + "/" + p;
}

mtd_status replay_records(mtd_ctx *c, const std::vector<HillRec> &recs) {
    if (recs.empty()) return MTD_OK;
    if (c->nb) return list_add_hills(c, recs);
    HillRec *d = nullptr;
    MTD_CU(dalloc(&d, sizeof(HillRec) * recs.size()), "replay");
    cudaMemcpy(d, recs.data(), sizeof(HillRec) * recs.size(), cudaMemcpyHostToDevice);
    if (c->plan_dirty) {
        build_plan(c);
        cudaMemcpy(c->d_plan, &c->plan, sizeof(BiasPlan), cudaMemcpyHostToDevice);
        c->plan_dirty = false;
    }
    launch_hills_replay(c->d_plan, d, (int)recs.size(), (int)c->grid_size, c->st);
    cudaError_t e = cudaStreamSynchronize(c->st);
    cudaFree(d);
    return cuda_check(c, e, "HILLS replay");
}

// HILLS rows `step cv[D] height sigma`; '#' and blank lines skipped, any
// other line that does not parse stops the restart with MTD_ERR_IO
// (GH_t0_uniformGrid.cu:101-192 on one rank).
mtd_status read_hills(mtd_ctx *c, const std::string &path, std::vector<HillRec> &recs, bool *exists) {
    FILE *f = std::fopen(path.c_str(), "r");
    if (exists) *exists = f != nullptr;
    if (!f) return MTD_OK;
    char line[1024];
    const int D = c->cfg.cv_dim;
    while (std::fgets(line, sizeof(line), f)) {
        const char *q = line;
        while (*q == ' ' || *q == '\t') ++q;
        if (*q == '#' || *q == '\n' || *q == '\r' || *q == '\0') continue;   // comment or blank line
        char *p = line, *e = nullptr;
        HillRec r{};
        r.step = std::strtoll(p, &e, 10);
        if (e == p) {
            std::fclose(f);
            return fail(c, MTD_ERR_IO, "malformed HILLS line (step is not an integer): " + std::string(line));
        }
        p = e;
        bool ok = true;
        for (int d = 0; d < D; ++d) {
            r.s[d] = std::strtod(p, &e);
            ok = ok && e != p;
            p = e;
        }
        r.w = std::strtod(p, &e);
        ok = ok && e != p;
        p = e;
        r.sigma = std::strtod(p, &e);
        ok = ok && e != p;
        if (!ok) {
            std::fclose(f);
            return fail(c, MTD_ERR_IO, "malformed HILLS line: " + std::string(line));
        }
        recs.push_back(r);
    }
    std::fclose(f);
    return MTD_OK;
}

}  // namespace ctx
}  // namespace mtd

extern "C" {

mtd_status mtd_hills_replay(mtd_ctx *c, const char *path) {
    if (!c || !path) return MTD_ERR_INVALID_ARG;
    if (!c->initialized) {
        mtd_status s = mtd_init(c);
        if (s != MTD_OK) return s;
    }
    std::vector<HillRec> recs;
    bool exists = false;
    mtd_status s = read_hills(c, path_in(c, path), recs, &exists);
    if (s != MTD_OK) return s;
    if (!exists) return fail(c, MTD_ERR_IO, std::string("cannot open ") + path);
    return replay_records(c, recs);
}

mtd_status mtd_get_grid(mtd_ctx *c, double *out, int64_t count) {
    if (!c || !out) return MTD_ERR_INVALID_ARG;
    if (!c->initialized || count != c->grid_size) return fail(c, MTD_ERR_INVALID_ARG, "grid not allocated or size mismatch");
    MTD_CU(cudaStreamSynchronize(c->st), "grid");
    MTD_CU(cudaMemcpy(out, c->d_grid, sizeof(double) * (size_t)count, cudaMemcpyDeviceToHost), "grid");
    return MTD_OK;
}

mtd_status mtd_nn_state(const mtd_ctx *c, int *hills, int *hills_fitted, int *usable) {
    if (!c) return MTD_ERR_INVALID_ARG;
    if (hills) *hills = c->nb ? mtd_nnbias_num_hills(c->nb) : 0;
    if (hills_fitted) *hills_fitted = c->h_fit;
    if (usable) *usable = c->nn_usable ? 1 : 0;
    return MTD_OK;
}

}  // extern "C"
