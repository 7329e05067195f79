// peratom.cu -- per-atom exports for `compute metad/atom` / Fix::extract
// (per-atom CV values, the exact dCV/dx), atom types for the chemical
// structure factor, and neighbour-list reporting.
#include "context.h"

#include <algorithm>

extern "C" {

mtd_status mtd_get_peratom(mtd_ctx *c, const char *key, double *out) {
    if (!c) return MTD_ERR_INVALID_ARG;
    return mtd_extract_peratom(c, key, out, c->n);
}

// dCV/dx of CAL `cal` at the last step's positions, into c->h_dcv ([n][3],
// caller order). The CV is the one the first SYMBOL on that CAL selects; the
// force kernels run once more with chain factor 1 on that symbol, 0 on the
// others and a zero input force, so their output is -dCV/dx (the exact
// gradient, every neighbour term included). Cached per step and CAL, as
// STEIN_QL::get_peratom_ptr caches per timestep (src/cvs/CVs_Steinhardt.cu:1278-1321).
static mtd_status dcvdx(mtd_ctx *c, const std::string &cal) {
    if (c->step_gen == 0) return fail(c, MTD_ERR_INVALID_ARG, "no step has run");
    if (c->dcv_gen == c->step_gen && c->dcv_cal == cal) return MTD_OK;
    int sym = -1;
    for (size_t q = 0; q < c->cfg.symbols.size() && sym < 0; ++q)
        if (c->cfg.symbols[q].cal == cal) sym = (int)q;
    if (sym < 0) return fail(c, MTD_ERR_INVALID_ARG, "dcvdx: no SYMBOL uses CAL " + cal);
    const int n = c->n;
    if (n > c->dcv_cap) {
        dfree(c->d_dcv);
        c->dcv_cap = 0;
        MTD_CU(dalloc(&c->d_dcv, sizeof(double) * 6 * (size_t)n), "dcvdx buffers");
        c->dcv_cap = n;
    }
    double *zero = c->d_dcv, *grad = c->d_dcv + 3 * (size_t)c->dcv_cap;
    MTD_CU(cudaMemsetAsync(zero, 0, sizeof(double) * 3 * (size_t)n, c->st), "dcvdx");
    const int launches = c->launches;
    launch_symbol_coef(c->d_plan, sym, c->d_ws1, c->st);
    if (c->fp64) run_forces<double>(c, c->last_sys, c->last_grid, c->last_x, c->last_mask, zero, grad, false);
    else run_forces<float>(c, c->last_sys, c->last_grid, c->last_x, c->last_mask, zero, grad, false);
    c->launches = launches;
    MTD_CU(cudaGetLastError(), "kernel launch");
    c->h_dcv.resize(3 * (size_t)n);
    MTD_CU(cudaMemcpyAsync(c->h_dcv.data(), grad, sizeof(double) * 3 * (size_t)n, cudaMemcpyDeviceToHost, c->st),
           "dcvdx");
    MTD_CU(cudaStreamSynchronize(c->st), "dcvdx");
    for (double &v : c->h_dcv) v = -v;
    c->dcv_gen = c->step_gen;
    c->dcv_cal = cal;
    return MTD_OK;
}

// The last step's neighbour lists of CAL `cal`, in caller order: kept[i] the
// neighbours the CV uses (for STEINH Q those inside the cutoff_Natoms cap),
// inrc[i] the neighbours inside the list criterion before the cap, and, when
// `lists` is given, the caller indices of the kept neighbours in ascending order.
static mtd_status host_lists(mtd_ctx *c, const std::string &cal, std::vector<int> &kept, std::vector<int> &inrc,
                             std::vector<std::vector<int>> *lists) {
    const Env *env = nullptr;
    for (const Unit &u : c->units)
        for (const std::string &cn : u.calnames)
            if (cn == cal && u.env >= 0) env = &c->envs[u.env];
    if (!env) return fail(c, MTD_ERR_INVALID_ARG, "no neighbour list for CAL " + cal);
    if (c->step_gen == 0) return fail(c, MTD_ERR_INVALID_ARG, "no step has run");
    const int n = c->n, M = env->M;
    const size_t stride = (size_t)c->cap_n;
    MTD_CU(cudaStreamSynchronize(c->st), "neighbour lists");
    std::vector<int> perm(n), cnt(n), raw;
    if (n > 0) {
        MTD_CU(cudaMemcpy(perm.data(), c->perm, sizeof(int) * n, cudaMemcpyDeviceToHost), "perm");
        MTD_CU(cudaMemcpy(cnt.data(), env->count, sizeof(int) * n, cudaMemcpyDeviceToHost), "neighbour counts");
        raw.resize((size_t)M * stride);
        MTD_CU(cudaMemcpy(raw.data(), env->list, sizeof(int) * raw.size(), cudaMemcpyDeviceToHost), "neighbour lists");
    }
    kept.assign(n, 0);
    inrc.assign(n, 0);
    if (lists) lists->assign(n, std::vector<int>());
    const int low = (1 << kFlagBit) - 1;
    for (int k = 0; k < n; ++k) {
        const int i = perm[k];
        const int m = std::min(cnt[k], M);
        inrc[i] = cnt[k];
        int nk = 0;
        for (int t = 0; t < m; ++t) {
            const int e = raw[(size_t)t * stride + k];
            if (env->kind == ENV_Q && !(e & (1 << kFlagBit))) continue;
            ++nk;
            if (lists) (*lists)[i].push_back(perm[e & low]);
        }
        kept[i] = nk;
        if (lists) std::sort((*lists)[i].begin(), (*lists)[i].end());
    }
    return MTD_OK;
}

mtd_status mtd_neighbor_stats(mtd_ctx *c, int64_t *rebuilds, int *skin_active) {
    if (!c) return MTD_ERR_INVALID_ARG;
    SkinState sk{};
    if (c->d_skin) {
        MTD_CU(cudaStreamSynchronize(c->st), "neighbour statistics");
        MTD_CU(cudaMemcpy(&sk, c->d_skin, sizeof(SkinState), cudaMemcpyDeviceToHost), "neighbour statistics");
    }
    if (rebuilds) *rebuilds = sk.builds;
    if (skin_active) *skin_active = c->skin_last ? 1 : 0;
    return MTD_OK;
}

mtd_status mtd_set_host_copy_mode(mtd_ctx *c, int mode) {
    if (!c || mode < 0 || mode > 3) return MTD_ERR_INVALID_ARG;
    c->host_copy_mode = mode;
    if (mode == 0) {   // time the modes again
        c->copy_pick = 0;
        c->copy_calls = 0;
        for (int k = 0; k < 4; ++k) {
            c->copy_ms[k] = 0.0;
            c->copy_cnt[k] = 0;
        }
    }
    return MTD_OK;
}

mtd_status mtd_host_copy_mode_in_use(mtd_ctx *c, int *mode) {
    if (!c || !mode) return MTD_ERR_INVALID_ARG;
    *mode = c->host_copy_mode ? c->host_copy_mode : c->copy_pick;
    return MTD_OK;
}

mtd_status mtd_neighbor_set_wait(mtd_ctx *c, int limit, int stall) {
    if (!c || limit < 0) return MTD_ERR_INVALID_ARG;
    c->rebuild_limit = limit > 0 ? limit : (1 << 22);
    c->rebuild_stall = stall ? 1 : 0;
    return MTD_OK;
}

mtd_status mtd_get_neighbors(mtd_ctx *c, const char *cal, int n, int *counts, int *idx, int max_per_atom) {
    if (!c || !cal || !counts || n < 0 || (idx && max_per_atom < 0)) return MTD_ERR_INVALID_ARG;
    if (n != c->n) return fail(c, MTD_ERR_INVALID_ARG, "atom count differs from the last step");
    std::vector<int> kept, inrc;
    std::vector<std::vector<int>> lists;
    const mtd_status s = host_lists(c, cal, kept, inrc, idx ? &lists : nullptr);
    if (s != MTD_OK) return s;
    for (int i = 0; i < n; ++i) {
        counts[i] = kept[i];
        if (!idx) continue;
        if (kept[i] > max_per_atom)
            return fail(c, MTD_ERR_INVALID_ARG, "atom " + std::to_string(i) + " has " + std::to_string(kept[i]) +
                                                    " neighbours, more than max_per_atom");
        for (int t = 0; t < max_per_atom; ++t) idx[(size_t)i * max_per_atom + t] = t < kept[i] ? lists[i][t] : -1;
    }
    return MTD_OK;
}

mtd_status mtd_extract_peratom(mtd_ctx *c, const char *key, double *out, int n) {
    if (!c || !key || !out) return MTD_ERR_INVALID_ARG;
    std::string k(key);
    if (k.rfind("colvar_peratom:", 0) == 0) k = k.substr(15);
    size_t dot = k.find('.');
    if (dot == std::string::npos) return fail(c, MTD_ERR_INVALID_ARG, "key must be <CAL>.<prop>");
    const std::string cal = k.substr(0, dot), prop = k.substr(dot + 1);
    if (n != c->n) return fail(c, MTD_ERR_INVALID_ARG, "atom count differs from the last step");
    MTD_CU(cudaStreamSynchronize(c->st), "extract");
    if (prop == "dcvdx_x" || prop == "dcvdx_y" || prop == "dcvdx_z") {
        mtd_status s = dcvdx(c, cal);
        if (s != MTD_OK) return s;
        const int a = prop.back() - 'x';
        for (int t = 0; t < n; ++t) out[t] = c->h_dcv[3 * (size_t)t + a];
        return MTD_OK;
    }
    if (prop == "nnb" || prop == "nrc") {   // neighbour counts (src/cvs/CVs_Steinhardt.cu:1324-1406)
        std::vector<int> kept, inrc;
        const mtd_status s = host_lists(c, cal, kept, inrc, nullptr);
        if (s != MTD_OK) return s;
        for (int t = 0; t < n; ++t) out[t] = prop == "nnb" ? kept[t] : inrc[t];
        return MTD_OK;
    }
    for (Unit &u : c->units) {
        for (size_t slot = 0; slot < u.calnames.size(); ++slot) {
            if (u.calnames[slot] != cal) continue;
            std::vector<int> perm(n);
            MTD_CU(cudaMemcpy(perm.data(), c->perm, sizeof(int) * n, cudaMemcpyDeviceToHost), "perm");
            std::vector<double> v(n, 0.0);
            const size_t R = real_size(c);
            std::vector<unsigned char> raw;
            int stride = 1, off = 0;
            const void *src = nullptr;
            if (prop == "stein_q" && u.kind == CAL_STEINH_Q) { src = u.Q; }
            else if (prop == "stein_q" && u.kind == CAL_STEINH_L) { src = u.lqs; stride = 2; off = (int)slot; }
            else if (prop == "stru_f" && u.kind == CAL_STRU_FACTOR && !u.wchem) { src = u.S; }
            else if (prop == "chem_pair_r" && u.kind == CAL_STRU_FACTOR && u.wchem) { src = u.S; }
            else return fail(c, MTD_ERR_INVALID_ARG, "unknown per-atom property " + prop + " for CAL " + cal);
            raw.resize(R * stride * (size_t)n);
            MTD_CU(cudaMemcpy(raw.data(), src, R * stride * (size_t)n, cudaMemcpyDeviceToHost), "extract");
            for (int t = 0; t < n; ++t) {
                double val = c->fp64 ? ((const double *)raw.data())[t * stride + off]
                                     : (double)((const float *)raw.data())[t * stride + off];
                out[perm[t]] = val;
            }
            return MTD_OK;
        }
    }
    return fail(c, MTD_ERR_INVALID_ARG, "unknown CAL " + cal);
}

mtd_status mtd_set_types(mtd_ctx *c, int n, const int *types) {
    if (!c || n < 0 || (n > 0 && !types)) return MTD_ERR_INVALID_ARG;
    if (n > c->types_cap) {
        dfree(c->d_types);
        c->types_cap = 0;
        MTD_CU(dalloc(&c->d_types, sizeof(int) * (size_t)(n + n / 4 + 1)), "atom types");
        c->types_cap = n + n / 4 + 1;
    }
    int maxt = 0;
    for (int i = 0; i < n; ++i) {
        if (types[i] < 0) return fail(c, MTD_ERR_INVALID_ARG, "atom types must be >= 0");
        maxt = std::max(maxt, types[i]);
    }
    MTD_CU(cudaStreamSynchronize(c->st), "atom types");   // no step in flight reads the old types
    if (n > 0) MTD_CU(cudaMemcpy(c->d_types, types, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice), "atom types");
    // type-weight tables (Stru_fact_chem_env constructor, src/cvs/CVs_Strufactor_chem.cu:33-55):
    // Chem_map value, else a Gaussian in the type index around Chem_ctarget; type 0 weighs 0
    for (Unit &u : c->units) {
        if (!u.chem) continue;
        std::vector<double> tab((size_t)maxt + 1);
        for (int t = 0; t <= maxt; ++t) {
            const double dt = t - u.chem_ctarget;
            tab[t] = std::exp(-dt * dt / (2.0 * u.chem_sigma * u.chem_sigma));
            for (const auto &kv : u.chem_map)
                if (kv.first == t) tab[t] = kv.second;
        }
        tab[0] = 0.0;
        if ((int)tab.size() > u.ntab) {
            dfree(u.d_wtab);
            u.ntab = 0;
            MTD_CU(dalloc(&u.d_wtab, sizeof(double) * tab.size()), "type weights");
        }
        u.ntab = (int)tab.size();
        MTD_CU(cudaMemcpy(u.d_wtab, tab.data(), sizeof(double) * tab.size(), cudaMemcpyHostToDevice), "type weights");
    }
    c->types_n = n;
    return MTD_OK;
}

int mtd_needs_types(const mtd_ctx *c) {
    if (!c) return 0;
    for (const Unit &u : c->units)
        if (u.chem) return 1;
    return 0;
}

int mtd_max_neighbors(mtd_ctx *c, const char *name) {
    if (!c || !name) return -1;
    for (Unit &u : c->units)
        for (auto &cn : u.calnames)
            if (cn == name && u.env >= 0) {
                const Env &e = c->envs[u.env];
                if (c->n == 0) return 0;
                std::vector<int> cnt(c->n);
                cudaStreamSynchronize(c->st);
                if (cudaMemcpy(cnt.data(), e.count, sizeof(int) * c->n, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
                int m = 0;
                for (int v : cnt) m = v > m ? v : m;
                return m;
            }
    return -1;
}

}  // extern "C"
