// context.cu -- the C ABI of libmetad_b200.so: context set-up from the
// `fix metad` arguments, device memory, the per-step launch sequence and the
// collection of each step's outputs (the other parts of the context live in
// decomp.cu, hills.cu, autotune.cu, peratom.cu and walkers.cu; context.h).
//
// Per step (one CUDA stream, no host synchronisation inside the step):
//   cells -> neighbour lists (one per distinct environment) -> CV value
//   kernels -> bias kernel (reductions, DIM, deposit, V, dV/ds) -> force
//   kernels (f_out = f_in - dV/dx) -> virial reduction.
// This is FixMetadynamics::post_force (src/core/fix_crystallize.cu:386-472)
// without its host loops, PCIe round trips and per-call synchronisations.
#include "context.h"

#include <algorithm>
#include <chrono>

namespace {
thread_local Prof *g_prof = nullptr;
thread_local bool g_pdl = false;
}

namespace mtd {
void pdl_set(bool on) { g_pdl = on; }
bool pdl_on() { return g_pdl; }
void prof_set(Prof *p) { g_prof = p; }
Prof *prof_get() { return g_prof; }
void prof_mark(const char *name, cudaStream_t st) {
    Prof *p = g_prof;
    if (!p || !p->on || p->n >= kProfMax) return;
    p->name[p->n] = name;
    cudaEventRecord(p->ev[p->n], st);
    ++p->n;
}
}  // namespace mtd

namespace mtd {
namespace ctx {

mtd_status fail(mtd_ctx *c, mtd_status s, const std::string &m) {
    if (c) c->err = m;
    return s;
}

mtd_status cuda_check(mtd_ctx *c, cudaError_t e, const char *what) {
    if (e == cudaSuccess) return MTD_OK;
    if (e == cudaErrorMemoryAllocation) return fail(c, MTD_ERR_OOM, std::string(what) + ": " + cudaGetErrorString(e));
    return fail(c, MTD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

size_t real_size(const mtd_ctx *c) { return c->fp64 ? sizeof(double) : sizeof(float); }

int record_stride(const mtd_ctx *c, const Unit &u) {
    if (u.kind == CAL_STEINH_L) return local_record_stride(u.LA, u.LB, c->fp64 ? 1 : 0);
    if (u.kind == CAL_STEINH_Q) return pad4(2 * (u.LA + 1));
    return 0;
}

double env_cutoff(const Env &e) { return e.rc; }

void use_slot(mtd_ctx *c, int k) {
    OutSlot &o = c->h_slots[k];
    c->h_out = o.out;
    c->h_status = &o.status;
    c->h_vir = o.vir;
    c->h_nhills = &o.nhills;
}

CellGrid make_grid(const mtd_ctx *c, double extra) {
    CellGrid g{};
    double rmax = 0.0;
    for (const Env &e : c->envs) rmax = std::fmax(rmax, env_cutoff(e) + extra);
    double Lmax = 0.0;
    for (int d = 0; d < 3; ++d) Lmax = std::fmax(Lmax, c->hi[d] - c->lo[d]);
    const double guard = 1e-6 * Lmax + 1e-6;
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
        double L = c->hi[d] - c->lo[d];
        if (!(L > 0)) L = 1.0;
        int nc = rmax > 0 ? (int)std::floor(L / (rmax + guard)) : 1;
        if (nc < 1) nc = 1;
        if (nc > 512) nc = 512;
        g.nc[d] = nc;
        g.periodic[d] = c->periodic[d];
        g.L[d] = L;
        g.invL[d] = 1.0 / L;
        g.lo[d] = c->lo[d];
        g.h[d] = L / nc;
        g.inv_h[d] = nc / L;
        g.hf[d] = (float)(L / nc);
        g.Lf[d] = (float)L;
        g.invLf[d] = 1.0f / (float)L;
        ncell *= nc;
    }
    // tiles of 4 x 4 x 4 cells where the fast neighbour search applies (every
    // periodic side with at least three cells)
    g.tiled = 1;
    for (int d = 0; d < 3; ++d)
        if (g.periodic[d] && g.nc[d] < 3) g.tiled = 0;
    if (g.tiled) {
        ncell = 64;
        for (int d = 0; d < 3; ++d) {
            g.nt[d] = (g.nc[d] + 3) / 4;
            ncell *= g.nt[d];
        }
    }
    g.ncell = (int)ncell;
    return g;
}

static bool same_grid(const CellGrid &a, const CellGrid &b) {
    for (int d = 0; d < 3; ++d)
        if (a.nc[d] != b.nc[d] || a.periodic[d] != b.periodic[d] || a.L[d] != b.L[d] || a.lo[d] != b.lo[d])
            return false;
    return true;
}

bool skin_grid(const mtd_ctx *c, CellGrid &g) {
    const double skin = c->cfg.neigh_skin;
    if (skin > 0.0 && !c->envs.empty()) {
        double rmax = 0.0;
        for (const Env &e : c->envs) rmax = std::fmax(rmax, env_cutoff(e) + skin);
        g = make_grid(c, skin);
        bool ok = true;
        for (int d = 0; d < 3; ++d)
            if (g.periodic[d] && (g.nc[d] < 3 || g.L[d] < 2.0 * rmax)) ok = false;
        if (ok) return true;
    }
    g = make_grid(c);
    return false;
}

// Neighbour criterion of an environment; the FP32 band [lo2, hi2] around the
// bound (2e-5 relative + 1e-4 A^2) is wide against the ~1e-6 A error of the
// cell-relative FP32 displacements, so outside it FP32 decides exactly.
NeighSpec neigh_spec(const Env &e) {
    NeighSpec ns{};
    ns.rc2 = e.rc * e.rc;
    ns.eps = e.eps;
    ns.sw = e.sw;
    ns.cap = e.kind == ENV_Q ? e.cap : 0;
    double eff = ns.rc2;
    if (e.kind == ENV_L && e.sw.type == SW_STEP) {
        ns.kind = NK_STEP;
        ns.r0 = e.sw.r0;
        eff = std::fmin(eff, e.sw.r0 * e.sw.r0);
    } else if (e.kind == ENV_L) {
        ns.kind = NK_SWITCH;
    } else {
        ns.kind = NK_RANGE;
    }
    ns.lo2 = (float)(eff * (1.0 - 2e-5) - 1e-4);
    ns.hi2 = (float)(ns.kind == NK_SWITCH ? ns.rc2 * (1.0 + 2e-5) + 1e-4 : eff * (1.0 + 2e-5) + 1e-4);
    return ns;
}

int estimate_M(const mtd_ctx *c, double rc, int n) {
    double V = 1.0;
    for (int d = 0; d < 3; ++d) V *= std::fmax(c->hi[d] - c->lo[d], 1e-9);
    const double rho = n / V;
    const double expect = 4.0 / 3.0 * kPi * rc * rc * rc * rho;
    int M = (int)std::ceil(1.6 * expect + 8.0);
    M = (M + 3) & ~3;
    return M < 8 ? 8 : M;
}

mtd_status alloc_cand(mtd_ctx *c, Env &e, int npad) {
    dfree(e.cand);
    dfree(e.ccount);
    MTD_CU(dalloc(&e.cand, sizeof(int) * (size_t)e.Mc * npad), "skin candidates");
    MTD_CU(dalloc(&e.ccount, sizeof(int) * (size_t)npad), "skin candidates");
    c->skin_valid = false;
    return MTD_OK;
}

mtd_status alloc_env(mtd_ctx *c, Env &e, int npad) {
    dfree(e.list);
    dfree(e.count);
    dfree(e.key_r2);
    dfree(e.key_id);
    dfree(e.nkept);
    MTD_CU(dalloc(&e.list, sizeof(int) * (size_t)e.M * npad), "neighbour list");
    MTD_CU(dalloc(&e.count, sizeof(int) * (size_t)npad), "neighbour counts");
    if (e.kind == ENV_Q) {
        MTD_CU(dalloc(&e.key_r2, sizeof(double) * (size_t)npad), "cap keys");
        MTD_CU(dalloc(&e.key_id, sizeof(int) * (size_t)npad), "cap keys");
        MTD_CU(dalloc(&e.nkept, sizeof(int) * (size_t)npad), "cap counts");
    }
    e.cap_n = npad;
    return MTD_OK;
}

mtd_status alloc_unit(mtd_ctx *c, Unit &u, int npad) {
    const size_t R = real_size(c);
    const int SQ = record_stride(c, u);
    const int nb = (npad + kBlock - 1) / kBlock;
    void **arrs[] = {&u.q, &u.nf, &u.lq, &u.lqs, &u.e12, &u.lam, &u.g, &u.tu, &u.Q, &u.S, &u.w};
    for (void **a : arrs) dfree(*a);
    dfree(u.partials);
    if (u.kind == CAL_STEINH_L) {
        MTD_CU(dalloc(&u.q, R * SQ * (size_t)npad), "q_lm");
        MTD_CU(dalloc(&u.lq, R * SQ * (size_t)npad), "LQ_lm");
        MTD_CU(dalloc(&u.lam, R * SQ * (size_t)npad), "adjoint");
        MTD_CU(dalloc(&u.nf, R * (size_t)npad), "NF");
        MTD_CU(dalloc(&u.lqs, R * 2 * (size_t)npad), "LQ");
        MTD_CU(dalloc(&u.e12, R * 4 * (size_t)npad), "weights");
        if (u.dsig) {
            MTD_CU(dalloc(&u.g, R * SQ * (size_t)npad), "G");
            MTD_CU(dalloc(&u.tu, R * 4 * (size_t)npad), "t,u");
        }
        u.nblocks = nb;
        MTD_CU(dalloc(&u.partials, sizeof(double) * 8 * (size_t)nb), "partials");
    } else if (u.kind == CAL_STEINH_Q) {
        MTD_CU(dalloc(&u.q, R * SQ * (size_t)npad), "q_lm");
        MTD_CU(dalloc(&u.Q, R * (size_t)npad), "Q");
        u.nblocks = nb;
        MTD_CU(dalloc(&u.partials, sizeof(double) * 8 * (size_t)nb), "partials");
    } else if (u.kind == CAL_STRU_FACTOR) {
        MTD_CU(dalloc(&u.S, R * (size_t)npad), "S");
        if (u.chem) MTD_CU(dalloc(&u.w, R * (size_t)npad), "type weights");
        u.nblocks = nb;
        MTD_CU(dalloc(&u.partials, sizeof(double) * 8 * (size_t)nb), "partials");
    } else {
        u.nblocks = sk_blocks(npad);
        MTD_CU(dalloc(&u.partials, sizeof(double) * (size_t)u.nblocks * (2 * u.K + 2)), "S(k) partials");
    }
    u.cap_n = npad;
    return MTD_OK;
}

cudaError_t h2d_pieces(void *dst, const void *src, size_t bytes, cudaStream_t st) {
    constexpr size_t kPiece = size_t(3) << 20;
    const size_t pieces = (bytes + kPiece - 1) / kPiece;
    for (size_t p = 0; p < pieces; ++p) {
        const size_t a = bytes * p / pieces, b = bytes * (p + 1) / pieces;
        const cudaError_t e = cudaMemcpyAsync(static_cast<char *>(dst) + a, static_cast<const char *>(src) + a, b - a,
                                              cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

mtd_status ensure_capacity(mtd_ctx *c, int n) {
    const int npad = ((n + kBlock - 1) / kBlock) * kBlock + kBlock;
    c->n = n;
    c->npad = npad;
    if (n != c->n_plan) {   // the bias kernel reads ceil(n / block) partials per unit
        c->plan_dirty = true;
        c->n_plan = n;
    }
    if (npad > c->cap_n) {
        const int cap = npad + npad / 4;
        dfree(c->d_x); dfree(c->d_fin); dfree(c->d_fout); dfree(c->d_mask); dfree(c->d_image);
        dfree(c->cellof); dfree(c->slot); dfree(c->perm); dfree(c->iperm); dfree(c->smask); dfree(c->arrival);
        dfree(c->xs); dfree(c->pf); dfree(c->d_vpart);
        MTD_CU(dalloc(&c->d_x, sizeof(double) * 3 * (size_t)cap), "x");
        MTD_CU(dalloc(&c->d_fin, sizeof(double) * 3 * (size_t)cap), "f");
        MTD_CU(dalloc(&c->d_fout, sizeof(double) * 3 * (size_t)cap), "f");
        MTD_CU(dalloc(&c->d_mask, sizeof(int) * (size_t)cap), "mask");
        MTD_CU(dalloc(&c->d_image, sizeof(int) * (size_t)cap), "image");
        MTD_CU(dalloc(&c->cellof, sizeof(int) * (size_t)cap), "cells");
        MTD_CU(dalloc(&c->slot, sizeof(int) * (size_t)cap), "cells");
        MTD_CU(dalloc(&c->perm, sizeof(int) * (size_t)cap), "perm");
        MTD_CU(dalloc(&c->iperm, sizeof(int) * (size_t)cap), "perm");
        MTD_CU(dalloc(&c->arrival, sizeof(int) * (size_t)cap), "cells");
        MTD_CU(dalloc(&c->smask, sizeof(int) * (size_t)cap), "mask");
        MTD_CU(dalloc(&c->xs, sizeof(double) * 3 * (size_t)cap), "x sorted");
        MTD_CU(dalloc(&c->pf, sizeof(float4) * (size_t)cap), "x float");
        c->cap_vpart = 8 * ((cap + 255) / 256) * (int)(c->units.size() + 1);
        MTD_CU(dalloc(&c->d_vpart, sizeof(double) * 8 * (size_t)c->cap_vpart), "virial partials");
        c->cap_n = cap;
        const bool skin = c->cfg.neigh_skin > 0.0 && !c->envs.empty();
        if (skin) {
            dfree(c->xref);
            MTD_CU(dalloc(&c->xref, sizeof(double) * 3 * (size_t)cap), "skin positions");
            if (!c->d_skin) {
                MTD_CU(dalloc(&c->d_skin, sizeof(SkinState)), "skin state");
                MTD_CU(cudaMemset(c->d_skin, 0, sizeof(SkinState)), "skin state");
                MTD_CU(dalloc(&c->d_rbar, sizeof(GridBar)), "rebuild barrier");
                MTD_CU(cudaMemset(c->d_rbar, 0, sizeof(GridBar)), "rebuild barrier");
            }
        }
        c->skin_valid = false;
        for (Env &e : c->envs) {
            if (e.M == 0) e.M = estimate_M(c, e.rc, n);
            if (e.kind == ENV_Q && e.M > 64) e.M = 64;
            mtd_status s = alloc_env(c, e, cap);
            if (s != MTD_OK) return s;
            if (skin) {
                if (e.Mc == 0) e.Mc = estimate_M(c, e.rc + c->cfg.neigh_skin, n);
                s = alloc_cand(c, e, cap);
                if (s != MTD_OK) return s;
            }
        }
        for (Unit &u : c->units) {
            mtd_status s = alloc_unit(c, u, cap);
            if (s != MTD_OK) return s;
        }
        c->plan_dirty = true;
    }
    return MTD_OK;
}

mtd_status ensure_cells(mtd_ctx *c, int ncell) {
    if (ncell + 1 > c->cap_cell) {
        dfree(c->count);
        dfree(c->start);
        const int cap = ncell + 1 + ncell / 4;
        MTD_CU(dalloc(&c->count, sizeof(int) * (size_t)cap), "cell counts");
        // zero once here; every build's scatter pass zeroes the counts it used
        MTD_CU(cudaMemset(c->count, 0, sizeof(int) * (size_t)cap), "cell counts");
        c->skin_valid = false;
        // ncell + 1 starts followed by the scan's per-block totals (1024-cell
        // blocks; 256-cell chunks in the persistent multi-walker step)
        MTD_CU(dalloc(&c->start, sizeof(int) * (size_t)(cap + 1 + cap / 256 + 2)), "cell starts");
        c->cap_cell = cap;
    }
    return MTD_OK;
}

mtd_status grow_lists(mtd_ctx *c, unsigned need, unsigned cand_need) {
    for (Env &e : c->envs) {
        if (need > 0 && e.M < (int)need) {
            if (e.kind == ENV_Q && need > 64)
                return fail(c, MTD_ERR_UNSUPPORTED, "STEINH Q: more than 64 atoms within cutoff_r");
            e.M = (((int)need + 8) + 3) & ~3;
            const mtd_status s = alloc_env(c, e, c->cap_n);
            if (s != MTD_OK) return s;
        }
        if (cand_need > 0 && e.Mc < (int)cand_need) {
            e.Mc = (((int)cand_need + 8) + 3) & ~3;
            const mtd_status s = alloc_cand(c, e, c->cap_n);   // the next step rebuilds
            if (s != MTD_OK) return s;
        }
    }
    return MTD_OK;
}

void build_plan(mtd_ctx *c) {
    BiasPlan &P = c->plan;
    const Config &cfg = c->cfg;
    P.D = cfg.cv_dim;
    for (int d = 0; d < 3; ++d) {
        if (d < P.D) {
            P.nbin[d] = cfg.dims[d].nbins;
            P.lo[d] = cfg.dims[d].lo;
            P.hi[d] = cfg.dims[d].hi;
            P.dcv[d] = (P.hi[d] - P.lo[d]) / P.nbin[d];
            P.band[d] = (int)std::ceil(4.0 * cfg.sigma / P.dcv[d]) + 1;   // GH_t0_uniformGrid.cu:87
        } else {
            P.nbin[d] = 1; P.lo[d] = 0; P.hi[d] = 1; P.dcv[d] = 1; P.band[d] = 0;
        }
    }
    P.sigma = cfg.sigma;
    P.h0 = cfg.height0;
    P.biasf = cfg.biasf;
    P.temp = cfg.temp;
    P.kb = c->boltz;
    P.wt = cfg.wt ? 1 : 0;
    P.pace = cfg.pace;
    P.nunit = (int)c->units.size();
    for (int u = 0; u < P.nunit; ++u) {
        const Unit &U = c->units[u];
        UnitPlan &Q = P.unit[u];
        Q.kind = U.kind;
        Q.coef = U.coef;
        if (U.kind == CAL_STRU_FACTOR_K) {
            Q.partials = nullptr;
            Q.nparts = 0;
            Q.pstride = 0;
            Q.nvals = 0;
            Q.rho = U.rho;
            Q.K = U.K;
            Q.sk_n = U.skn;
        } else {
            Q.partials = U.partials;
            Q.nparts = (c->n + kBlock - 1) / kBlock;
            Q.pstride = 8;
            Q.nvals = U.kind == CAL_STEINH_L ? 5 : 4;
            Q.rho = nullptr;
            Q.K = 0;
            Q.sk_n = nullptr;
        }
    }
    P.grid = c->d_grid;
    P.grid_size = c->d_grid ? c->grid_size : 0;
    P.hills = c->d_hills;
    P.hill_cap = kHillCap;
    P.nhills = c->d_nhills;
    P.out = c->d_out;
    P.status = c->d_status;
    P.save = c->d_ws1;
    P.gsum = c->nown >= 0 ? c->d_xchg : nullptr;
}

// Neighbour-list and CV-unit layout from the parsed CAL table (env pooling as in
// Steinhardt_env::get_or_create, src/cvs/CVs_Steinhardt.cu:191-220).
mtd_status plan_units(mtd_ctx *c) {
    Config &cfg = c->cfg;
    auto same_sw = [](const SwParams &a, const SwParams &b) {
        return a.type == b.type && a.r0 == b.r0 && a.d0 == b.d0 && a.alpha == b.alpha && a.n == b.n && a.m == b.m;
    };
    std::map<std::string, int> unit_of;   // CAL name -> unit
    std::map<std::string, int> slot_of;   // CAL name -> slot in unit
    for (auto &kv : cfg.cals) {
        const CalDef &d = kv.second;
        bool used = false;
        for (auto &s : cfg.symbols) used = used || (s.cal == d.name);
        if (d.kind == CAL_STRU_FACTOR_K) {
            Unit u;
            u.kind = d.kind;
            u.calnames = {d.name};
            u.groupbit = d.groupbit;
            u.K = d.nk;
            u.used = used;
            unit_of[d.name] = (int)c->units.size();
            slot_of[d.name] = 0;
            c->units.push_back(u);
            continue;
        }
        int ek = d.kind == CAL_STEINH_Q ? ENV_Q : (d.kind == CAL_STEINH_L ? ENV_L : ENV_R);
        int env = -1;
        for (size_t e = 0; e < c->envs.size(); ++e) {
            const Env &E = c->envs[e];
            if (E.kind != ek || E.rc != d.cutoff_r) continue;
            if (ek == ENV_Q && E.cap != d.cutoff_natoms) continue;
            if (ek == ENV_L && (!same_sw(E.sw, d.sw_r) || E.eps != d.cutoff_eps)) continue;
            env = (int)e;
        }
        if (env < 0) {
            Env E;
            E.kind = ek;
            E.rc = d.cutoff_r;
            E.cap = ek == ENV_Q ? d.cutoff_natoms : 0;
            E.sw = d.sw_r;
            E.eps = d.cutoff_eps;
            env = (int)c->envs.size();
            c->envs.push_back(E);
        }
        // fuse a second STEINH L order into an open unit of the same environment
        if (d.kind == CAL_STEINH_L) {
            bool fused = false;
            for (size_t u = 0; u < c->units.size(); ++u) {
                Unit &U = c->units[u];
                if (U.kind != CAL_STEINH_L || U.env != env || U.LB != 0 || U.groupbit != d.groupbit) continue;
                const int key = U.LA * 16 + d.l;
                if (key != 4 * 16 + 6 && key != 6 * 16 + 4 && key != 3 * 16 + 4 && key != 3 * 16 + 6) continue;
                U.LB = d.l;
                U.sw_cvB = d.sw_cv;
                U.calnames.push_back(d.name);
                U.used = U.used || used;
                unit_of[d.name] = (int)u;
                slot_of[d.name] = 1;
                fused = true;
                break;
            }
            if (fused) continue;
        }
        Unit u;
        u.kind = d.kind;
        u.calnames = {d.name};
        u.env = env;
        u.groupbit = d.groupbit;
        u.LA = d.l;
        u.LB = 0;
        u.sw_r = d.sw_r;
        u.sw_cvA = d.sw_cv;
        u.sw_cvB = d.sw_cv;
        u.dsig = (d.kind == CAL_STEINH_L) && d.sw_r.type != SW_STEP;
        u.rc = d.cutoff_r;
        u.qf = d.q_factor;
        u.sf_sw = d.sf_sw;
        u.chem = d.kind == CAL_STRU_FACTOR && d.chem;
        u.wchem = d.kind == CAL_STRU_FACTOR && d.wchem;
        u.chem_ctarget = d.chem_ctarget;
        u.chem_sigma = d.chem_sigma;
        u.chem_map = d.chem_map;
        u.used = used;
        unit_of[d.name] = (int)c->units.size();
        slot_of[d.name] = 0;
        c->units.push_back(u);
    }
    if ((int)c->units.size() > kMaxUnits) return fail(c, MTD_ERR_UNSUPPORTED, "too many CAL units");
    // symbols
    BiasPlan &P = c->plan;
    P.nsym = (int)cfg.symbols.size();
    for (int q = 0; q < P.nsym; ++q) {
        const SymbolDef &s = cfg.symbols[q];
        const CalDef &d = cfg.cals[s.cal];
        SymPlan sp{};
        sp.unit = unit_of[s.cal];
        sp.slot = slot_of[s.cal];
        Unit &U = c->units[sp.unit];
        if (d.kind == CAL_STEINH_Q) {
            if (s.func == "AVE") sp.kind = SYM_Q_AVE;
            else {
                sp.kind = SYM_Q_SW;
                int slot = -1;
                for (size_t t = 0; t < U.qswnames.size(); ++t)
                    if (U.qswnames[t] == s.sub) slot = (int)t;
                if (slot < 0) {
                    if (U.qsw.size() >= 2) return fail(c, MTD_ERR_UNSUPPORTED, "at most two SW_FUNC symbols per STEINH Q CAL");
                    U.qsw.push_back(cfg.sws[s.sub]);
                    U.qswnames.push_back(s.sub);
                    slot = (int)U.qsw.size() - 1;
                }
                sp.slot = slot;
            }
        } else if (d.kind == CAL_STEINH_L) {
            if (s.func == "MEAN_SOLID" || s.func == "AVE") sp.kind = SYM_L_MEAN;
            else if (s.func == "NSOLID" || s.func == "SW_FUNC") sp.kind = SYM_L_NSOLID;
            else sp.kind = SYM_L_FRAC;
            if (sp.slot == 0) U.sw_cvA = d.sw_cv;
            else U.sw_cvB = d.sw_cv;
        } else if (d.kind == CAL_STRU_FACTOR) {
            sp.kind = s.func == "AVE" ? SYM_SF_AVE : SYM_SF_COUNT;
        } else {
            sp.kind = SYM_SK_AVE;
        }
        P.sym[q] = sp;
        c->symnames.push_back(s.name);
    }
    for (int dd = 0; dd < cfg.cv_dim; ++dd) {
        std::vector<ExprInstr> code;
        std::string e = compile_expr(cfg.dims[dd].expr, c->symnames, code);
        if (!e.empty()) return fail(c, MTD_ERR_PARSE, e);
        P.ncode[dd] = (int)code.size();
        for (size_t t = 0; t < code.size(); ++t) P.code[dd][t] = code[t];
        c->code.push_back(code);
    }
    // per-unit small device blocks
    for (Unit &u : c->units) {
        MTD_CU(dalloc(&u.coef, sizeof(double) * 8), "coefficients");
        MTD_CU(cudaMemset(u.coef, 0, sizeof(double) * 8), "coefficients");
        if (u.kind == CAL_STRU_FACTOR_K) {
            const CalDef &d = cfg.cals[u.calnames[0]];
            MTD_CU(dalloc(&u.kvec, sizeof(double) * 3 * u.K), "k vectors");
            MTD_CU(dalloc(&u.rho, sizeof(double) * 2 * u.K), "rho");
            MTD_CU(dalloc(&u.skn, sizeof(double)), "rho");
            MTD_CU(cudaMemcpy(u.kvec, d.kvecs.data(), sizeof(double) * 3 * u.K, cudaMemcpyHostToDevice), "k vectors");
        }
    }
    return MTD_OK;
}

// Atoms that are centres of the CV sums: all of them, or under domain
// decomposition the caller's first nlocal (the rest are ghosts).
int owned(const mtd_ctx *c) { return c->nown >= 0 ? std::min(c->nown, c->n) : c->n; }

NeighDev env_dev(const Env &e) {
    NeighDev nd{};
    nd.list = e.list;
    nd.count = e.count;
    nd.key_r2 = e.key_r2;
    nd.key_id = e.key_id;
    nd.nkept = e.nkept;
    nd.M = e.M;
    return nd;
}

SysDev sys_dev(mtd_ctx *c, const double *x, const int *mask, const int *image) {
    SysDev s{};   // every field set (skin, xref: null unless the skin path sets them)
    s.n = c->n;
    s.npad = c->cap_n;
    s.x = x;
    s.mask = mask;
    s.image = image;
    s.cellof = c->cellof;
    s.slot = c->slot;
    s.count = c->count;
    s.start = c->start;
    s.perm = c->perm;
    s.iperm = c->iperm;
    s.arrival = c->arrival;
    s.smask = c->smask;
    s.xs = c->xs;
    s.pf = c->pf;
    s.nown = owned(c);
    s.status = c->d_status;
    return s;
}

template <typename T> LocalDev<T> local_dev(mtd_ctx *c, Unit &u, const CellGrid &g) {
    LocalDev<T> d{};
    d.n = c->n; d.npad = c->cap_n; d.SQ = record_stride(c, u); d.LA = u.LA; d.LB = u.LB;
    d.groupbit = u.groupbit; d.sw_r = u.sw_r; d.sw_cvA = u.sw_cvA; d.sw_cvB = u.sw_cvB;
    d.smask = c->smask; d.perm = c->perm; d.geo = make_geo<T>(g, c->pf, c->xs); d.nb = env_dev(c->envs[u.env]);
    d.q = (T *)u.q; d.nf = (T *)u.nf; d.lq = (T *)u.lq; d.lqs = (T *)u.lqs; d.e12 = (T *)u.e12;
    d.lam = (T *)u.lam; d.g = (T *)u.g; d.tu = (T *)u.tu; d.partials = u.partials; d.coef = u.coef;
    d.qblock = c->tune_q;
    d.lblock = c->tune_l;
    d.qsplit = c->tune_qsplit;
    return d;
}

template <typename T> GlobalDev<T> global_dev(mtd_ctx *c, Unit &u, const CellGrid &g) {
    GlobalDev<T> d{};
    d.n = c->n; d.npad = c->cap_n; d.SQ = record_stride(c, u); d.L = u.LA; d.groupbit = u.groupbit;
    d.nsw = (int)u.qsw.size();
    for (int t = 0; t < d.nsw; ++t) d.sw[t] = u.qsw[t];
    d.smask = c->smask; d.perm = c->perm; d.geo = make_geo<T>(g, c->pf, c->xs); d.exact = geo_d(g, c->xs);
    d.nb = env_dev(c->envs[u.env]);
    d.q = (T *)u.q; d.Q = (T *)u.Q; d.partials = u.partials; d.coef = u.coef;
    return d;
}

template <typename T> DebyeDev<T> debye_dev(mtd_ctx *c, Unit &u, const CellGrid &g) {
    DebyeDev<T> d{};
    d.n = c->n; d.npad = c->cap_n; d.groupbit = u.groupbit; d.rc2 = u.rc * u.rc; d.qf = u.qf; d.sw = u.sf_sw;
    d.smask = c->smask; d.perm = c->perm; d.geo = make_geo<T>(g, c->pf, c->xs); d.nb = env_dev(c->envs[u.env]);
    d.S = (T *)u.S; d.partials = u.partials; d.coef = u.coef;
    d.w = u.chem ? (T *)u.w : nullptr;
    d.types = c->d_types;
    d.wtab = u.d_wtab;
    d.ntab = u.ntab;
    return d;
}

SkDev sk_dev(mtd_ctx *c, Unit &u, const double *x, const int *mask) {
    SkDev d{};
    d.n = c->n; d.K = u.K; d.groupbit = u.groupbit; d.x = x; d.mask = mask; d.k = u.kvec;
    d.partials = u.partials; d.nblocks = u.nblocks; d.rho = u.rho; d.ngroup = u.skn; d.coef = u.coef;
    d.fp64 = c->fp64;
    d.nown = owned(c);
    d.qv = c->tune_skq;
    d.qf = c->tune_skqf;
    return d;
}

template <typename T> void run_values(mtd_ctx *c, const CellGrid &g, const double *x, const int *mask) {
    cudaStream_t st = c->st;
    for (Unit &u : c->units) {
        if (u.kind == CAL_STEINH_L) {
            LocalDev<T> d = local_dev<T>(c, u, g);
            if (c->skin_last && u.env >= 0 && u.env < (int)c->env_fused.size() && c->env_fused[u.env]) {
                // skin lists: this unit's q pass filters its candidates first
                const Env &e = c->envs[u.env];
                d.filter = 1;
                d.fgf = geo_f(g, c->pf);
                d.fgd = geo_d(g, c->xs);
                d.fspec = neigh_spec(e);
                d.cand = env_dev(e);
                d.cand.list = e.cand;
                d.cand.count = e.ccount;
                d.cand.M = e.Mc;
                d.status = c->d_status;
                d.reset = c->skin_reset_pending ? c->d_skin : nullptr;
                c->skin_reset_pending = false;
            }
            launch_local_values<T>(d, st);
            c->launches += 2;
        } else if (u.kind == CAL_STEINH_Q) {
            launch_global_values<T>(global_dev<T>(c, u, g), st);
            c->launches += 1;
        } else if (u.kind == CAL_STRU_FACTOR) {
            launch_debye_values<T>(debye_dev<T>(c, u, g), st);
            c->launches += u.chem ? 2 : 1;
        } else {
            launch_sk_values(sk_dev(c, u, x, mask), st);
            c->launches += 2;
        }
    }
}

// The deck's one force-producing unit when it is a STEINH L unit, else null.
Unit *single_local_unit(mtd_ctx *c) {
    Unit *only = nullptr;
    int used = 0;
    for (Unit &u : c->units)
        if (u.used) {
            ++used;
            only = &u;
        }
    return used == 1 && only->kind == CAL_STEINH_L ? only : nullptr;
}

// Forces: the first unit reads f_in, the later ones accumulate into f_out.
template <typename T>
void run_forces(mtd_ctx *c, const SysDev &s, const CellGrid &g, const double *x, const int *mask, const double *fin,
                double *fout, bool virial) {
    cudaStream_t st = c->st;
    // mtd_post_force on pinned host f (zero copy): the force pass runs over
    // caller indices, so each warp reads and writes one contiguous stretch
    // of the host array; the same per-atom arithmetic as the sorted order
    if (c->zc_on && !virial) {
        Unit *only = single_local_unit(c);
        LocalDev<T> d = local_dev<T>(c, *only, g);
        launch_local_lambda<T>(d, st);
        d.iperm = c->iperm;
        d.i0 = 0;
        d.i1 = c->n;
        launch_local_force_pass<T>(d, fin, fout, s, g, nullptr, c->d_status, st);
        c->launches += 2;
        return;
    }
    bool first = true;
    int voff = 0;
    for (Unit &u : c->units) {
        if (!u.used) continue;
        const double *src = first ? fin : fout;
        double *vp = virial ? c->d_vpart + (size_t)voff * 8 : nullptr;
        const int nb = (c->n + kBlock - 1) / kBlock;
        if (u.kind == CAL_STEINH_L) {
            launch_local_forces<T>(local_dev<T>(c, u, g), src, fout, s, g, vp, c->d_status, st);
            c->launches += 2;
        } else if (u.kind == CAL_STEINH_Q) {
            launch_global_forces<T>(global_dev<T>(c, u, g), src, fout, s, g, vp, c->d_status, st);
            c->launches += 1;
        } else if (u.kind == CAL_STRU_FACTOR) {
            launch_debye_forces<T>(debye_dev<T>(c, u, g), src, fout, s, g, vp, c->d_status, st);
            c->launches += 1;
        } else {
            launch_sk_forces(sk_dev(c, u, x, mask), src, fout, s, g, vp, st);
            c->launches += 1;
        }
        voff += nb;
        first = false;
    }
    if (first && fin != fout) cudaMemcpyAsync(fout, fin, sizeof(double) * 3 * (size_t)c->n, cudaMemcpyDeviceToDevice, st);
    if (virial) {
        launch_virial_finalize(c->d_vpart, voff, c->d_vir, st);
        c->launches += 1;
    }
}

// Adds the kernel intervals of the profiled steps in the buffer to the
// per-name totals (an interval ending at a step's "start" mark spans the gap
// between two steps and is not counted).  The marks of many steps are kept so
// that profiling does not make the host wait for every step.
void prof_collect(mtd_ctx *c) {
    Prof &p = c->prof;
    if (p.n >= 2) {
        cudaEventSynchronize(p.ev[p.n - 1]);
        for (int i = 1; i < p.n; ++i) {
            if (std::strcmp(p.name[i], "start") == 0) continue;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.ev[i - 1], p.ev[i]);
            auto &t = c->prof_total[p.name[i]];
            t.first += 1;
            t.second += ms;
        }
    }
    p.n = 0;
}


// Stage 1 of a step: capacity, plan, cell list, neighbour lists, CV values.
mtd_status enqueue_values(mtd_ctx *c, int n, const double *x, const int *mask, const int *image) {
    if (!c->box_set) return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_box must be called before the first step");
    mtd_status s0 = ensure_capacity(c, n);
    if (s0 != MTD_OK) return s0;
    if (c->nown > n)
        return fail(c, MTD_ERR_INVALID_ARG, "domain decomposition: nlocal " + std::to_string(c->nown) +
                                                " exceeds the " + std::to_string(n) + " atoms of this step");
    if (c->nown >= 0 && !c->d_xchg) {
        build_plan(c);
        c->xchg_n = unit_sums_count(c->plan);
        MTD_CU(dalloc(&c->d_xchg, sizeof(double) * (size_t)c->xchg_n), "domain totals");
        MTD_CU(cudaHostAlloc((void **)&c->h_xchg, sizeof(double) * (size_t)c->xchg_n, cudaHostAllocDefault),
               "domain totals");
        c->plan_dirty = true;
    }
    CellGrid g;
    const bool skin = skin_grid(c, g);
    c->last_grid = g;
    if (c->plan_dirty) {
        build_plan(c);
        MTD_CU(cudaMemcpyAsync(c->d_plan, &c->plan, sizeof(BiasPlan), cudaMemcpyHostToDevice, c->st), "plan");
        MTD_CU(cudaStreamSynchronize(c->st), "plan");
        c->plan_dirty = false;
    }
    SysDev s = sys_dev(c, x, mask, image);
    if (!c->envs.empty()) {
        mtd_status sc = ensure_cells(c, g.ncell);
        if (sc != MTD_OK) return sc;
        s.count = c->count;
        s.start = c->start;
        if (skin) {
            // kept sorted order and candidate lists: repack and test every
            // step, rebuild (the gated kernels) only when due, then filter
            // the candidates to the exact lists at the current positions
            const bool same = c->skin_valid && c->skin_n == n && same_grid(c->skin_grid, g);
            s.skin = c->d_skin;
            s.xref = c->xref;
            launch_refresh(g, s, c->cfg.neigh_every, 0.5 * c->cfg.neigh_skin, same ? 0 : 1, c->st);
            c->launches += 1;
            // the gated rebuild: cell list and the first environment's
            // candidates as one cooperative launch where it can run, else
            // the separate gated kernels
            // (inside a stream capture, e.g. the walkers' CUDA graph, the
            // separate gated kernels are captured instead)
            cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
            cudaStreamIsCapturing(c->st, &cap);
            const bool one = c->d_rbar && rebuild_blocks() > 0 && cap == cudaStreamCaptureStatusNone;
            if (!one) c->launches += launch_build_cells(g, s, c->st);
            for (size_t ei = 0; ei < c->envs.size(); ++ei) {
                Env &e = c->envs[ei];
                NeighSpec ns = neigh_spec(e);
                ns.variant = c->tune_nbr;
                ns.kind = NK_CAND;
                ns.cap = 0;
                const double rb = e.rc + c->cfg.neigh_skin;
                ns.hi2 = (float)(rb * rb * (1.0 + 2e-5) + 1e-4);
                NeighDev cd = env_dev(e);
                cd.list = e.cand;
                cd.count = e.ccount;
                cd.M = e.Mc;
                if (one && ei == 0) {
                    MTD_CU(launch_rebuild(g, s, ns, cd, c->d_status, c->d_rbar, c->rebuild_limit, c->rebuild_stall,
                                          c->st),
                           "skin-list rebuild");
                    c->rebuild_stall = 0;
                } else {
                    launch_neighbors(g, s, ns, cd, c->d_status, c->st);
                }
                c->launches += 1;
            }
            // an environment that only one STEINH L unit reads is filtered
            // inside that unit's q pass; the others by their own kernel
            c->env_fused.assign(c->envs.size(), 0);
            std::vector<int> users(c->envs.size(), 0);
            for (const Unit &u : c->units)
                if (u.env >= 0) users[u.env] += 1;
            for (const Unit &u : c->units)
                if (u.env >= 0 && u.kind == CAL_STEINH_L && users[u.env] == 1) c->env_fused[u.env] = 1;
            bool first = true;
            for (size_t ei = 0; ei < c->envs.size(); ++ei) {
                if (c->env_fused[ei]) continue;
                Env &e = c->envs[ei];
                const NeighSpec ns = neigh_spec(e);
                NeighDev cd = env_dev(e);
                cd.list = e.cand;
                cd.count = e.ccount;
                cd.M = e.Mc;
                launch_filter(g, s, ns, env_dev(e), cd, c->d_status, first ? c->d_skin : nullptr, c->st);
                first = false;
                c->launches += 1;
                if (ns.cap > 0) {
                    launch_select_cap(g, s, ns, env_dev(e), c->st);
                    c->launches += 1;
                }
            }
            c->skin_reset_pending = first;
            c->skin_valid = true;
            c->skin_n = n;
            c->skin_grid = g;
        } else {
            c->launches += launch_build_cells(g, s, c->st);
            for (Env &e : c->envs) {
                NeighSpec ns = neigh_spec(e);
                ns.variant = c->tune_nbr;
                launch_neighbors(g, s, ns, env_dev(e), c->d_status, c->st);
                c->launches += ns.cap > 0 ? 2 : 1;
            }
            c->skin_valid = false;
        }
        c->skin_last = skin;
    }
    for (const Unit &u : c->units)
        if (u.chem && c->types_n != n)
            return fail(c, MTD_ERR_INVALID_ARG,
                        "STRU_FACTOR Chemical needs the atom types of these " + std::to_string(n) +
                            " atoms: call mtd_set_types first");
    if (c->fp64) run_values<double>(c, g, x, mask);
    else run_values<float>(c, g, x, mask);
    c->last_sys = s;
    c->last_x = x;
    c->last_mask = mask;
    c->step_gen += 1;
    MTD_CU(cudaGetLastError(), "kernel launch");
    return MTD_OK;
}

// Stage 3 (after the bias kernel): forces, virial, outputs to pinned host memory.
mtd_status enqueue_forces(mtd_ctx *c, long long step, const double *x, const int *mask, const double *fin,
                          double *fout, bool virial) {
    if (c->fp64) run_forces<double>(c, c->last_sys, c->last_grid, x, mask, fin, fout, virial);
    else run_forces<float>(c, c->last_sys, c->last_grid, x, mask, fin, fout, virial);
    MTD_CU(cudaGetLastError(), "kernel launch");
    // outputs of this step into pinned host memory
    const int slot = c->ring ? c->slot_next : 0;
    use_slot(c, slot);
    MTD_CU(cudaMemcpyAsync(c->h_out, c->d_out, sizeof(double) * 64, cudaMemcpyDeviceToHost, c->st), "outputs");
    MTD_CU(cudaMemcpyAsync(c->h_status, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->st), "status");
    MTD_CU(cudaMemcpyAsync(c->h_nhills, c->d_nhills, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->st), "hills");
    if (virial) MTD_CU(cudaMemcpyAsync(c->h_vir, c->d_vir, sizeof(double) * 6, cudaMemcpyDeviceToHost, c->st), "virial");
    if (c->ring) {
        MTD_CU(cudaEventRecord(c->slot_ev[slot], c->st), "outputs");
        c->fifo.push_back(PendingOut{slot, step, virial});
        c->slot_next = (slot + 1) % kOutSlots;
        return MTD_OK;
    }
    c->want_virial = virial;
    c->pending = true;
    c->pending_step = step;
    return MTD_OK;
}

// f_ready (may be null): an event the force kernels wait for (forces uploaded
// on the side stream while the CV passes run).
mtd_status enqueue_step(mtd_ctx *c, long long step, int n, const double *x, const int *mask, const int *image,
                        const double *fin, double *fout, bool virial, cudaEvent_t f_ready) {
    ProfScope prof_scope(c);
    PdlScope pdl_scope;
    c->launches = 0;
    mtd_status s = enqueue_values(c, n, x, mask, image);
    if (s != MTD_OK) return s;
    if (c->nown >= 0) {
        s = exchange_totals(c);
        if (s != MTD_OK) return s;
    }
    if (c->nb) {   // hill-list bias: CVs, V and dV/ds at s, deposit and coefficients
        launch_list_cvs(c->d_plan, c->d_ws1, c->st);
        s = nnbias_enqueue_vdv(c->nb, c->d_out, c->d_vdv, c->nn_usable, c->h_fit, c->st);
        if (s != MTD_OK) return fail(c, s, mtd_nnbias_last_error(c->nb));
        launch_list_finish(c->d_plan, step, c->d_ws1, c->d_vdv, c->st);
        c->launches += 4;
    } else {
        launch_bias_step(c->d_plan, step, c->st);
        c->launches += 1;
    }
    if (f_ready) MTD_CU(cudaStreamWaitEvent(c->st, f_ready, 0), "force upload");
    return enqueue_forces(c, step, x, mask, fin, fout, virial);
}

// Collects the outputs of the last enqueued step (stream already synchronised).
mtd_status collect(mtd_ctx *c) {
    if (!c->pending) return MTD_OK;
    c->pending = false;
    const int D = c->cfg.cv_dim;
    for (int d = 0; d < D; ++d) c->cv[d] = c->h_out[d];
    c->bias = c->h_out[D];
    if (c->want_virial)
        for (int t = 0; t < 6; ++t) c->virial[t] = c->h_vir[t];
    const unsigned long long nh = *c->h_nhills;
    if (nh > c->hills_written) {
        unsigned long long from = c->hills_written;
        if (nh - from > (unsigned long long)kHillCap) from = nh - kHillCap;
        std::vector<HillRec> recs;
        if (nh - from == 1 && c->h_out[D + 1] != 0.0) {   // this step's hill, copied out with its outputs
            HillRec r;
            std::memcpy(&r, c->h_out + kOutHillOffset, sizeof(HillRec));
            write_hill_line(c, r);
            recs.push_back(r);
        } else {
            // the new records in at most two copies (the ring wraps once at most)
            recs.resize((size_t)(nh - from));
            const size_t a = (size_t)(from % kHillCap);
            const size_t first = std::min(recs.size(), (size_t)kHillCap - a);
            MTD_CU(cudaMemcpy(recs.data(), c->d_hills + a, sizeof(HillRec) * first, cudaMemcpyDeviceToHost),
                   "hill records");
            if (first < recs.size())
                MTD_CU(cudaMemcpy(recs.data() + first, c->d_hills, sizeof(HillRec) * (recs.size() - first),
                                  cudaMemcpyDeviceToHost),
                       "hill records");
            for (const HillRec &r : recs) write_hill_line(c, r);
        }
        c->hills_written = nh;
        if (c->nb) {
            mtd_status s = list_add_hills(c, recs);
            if (s != MTD_OK) return s;
        }
    }
    if (c->f_rec && c->cfg.rec_pace > 0 && c->pending_step % c->cfg.rec_pace == 0) {
        std::fprintf(c->f_rec, "%lld", c->pending_step);
        for (int d = 0; d < D; ++d) std::fprintf(c->f_rec, " %.16g", c->cv[d]);
        std::fprintf(c->f_rec, " %.16g\n", c->bias);
        std::fflush(c->f_rec);
    }
    if (c->h_status->bad_pos)
        return fail(c, MTD_ERR_NAN, "non-finite atom position (NaN or Inf): the step deposited nothing and applied no bias force");
    if (c->h_status->timeout) {
        // a grid-barrier wait of the one-launch skin-list rebuild ran out: the
        // device marked the skin state invalid (the next step rebuilds from
        // scratch); the barrier words are reset for the next rebuild
        if (c->d_rbar) MTD_CU(cudaMemsetAsync(c->d_rbar, 0, sizeof(GridBar), c->st), "rebuild barrier");
        return fail(c, MTD_ERR_TIMEOUT,
                    "neighbour-list rebuild: a grid-barrier wait ran out; the step deposited nothing and applied no "
                    "bias force, the next step rebuilds the lists");
    }
    if (c->h_status->nan_force) return fail(c, MTD_ERR_NAN, "STEIN_QL CV error: force is infinity, check your system or cv_value.");
    return MTD_OK;
}

// Collects enqueued steps in order: every step whose outputs have arrived
// (block: every step, waiting for each).  A step that overflowed a neighbour
// list deposited nothing and applied no bias force; it is not collected, and
// the overflow is kept for mtd_sync to report.
mtd_status drain(mtd_ctx *c, bool block) {
    while (!c->fifo.empty()) {
        const PendingOut p = c->fifo.front();
        if (block) {
            MTD_CU(cudaEventSynchronize(c->slot_ev[p.slot]), "step outputs");
        } else {
            const cudaError_t q = cudaEventQuery(c->slot_ev[p.slot]);
            if (q == cudaErrorNotReady) break;
            MTD_CU(q, "step outputs");
        }
        c->fifo.pop_front();
        use_slot(c, p.slot);
        if (c->h_status->overflow || c->h_status->cand_overflow) {
            c->overflow_seen = std::max(c->overflow_seen, c->h_status->overflow);
            c->overflow_cand_seen = std::max(c->overflow_cand_seen, c->h_status->cand_overflow);
            continue;
        }
        c->pending = true;
        c->pending_step = p.step;
        c->want_virial = p.virial;
        const mtd_status s = collect(c);
        if (s != MTD_OK) return s;
    }
    return MTD_OK;
}

// One walker's arguments for the persistent multi-walker step: the host part
// of enqueue_values and enqueue_forces (capacity, plan, cell arrays, the
// per-step lists' layout) with no launch.  The caller checked that the
// context has one STEINH L unit on one environment and no skin lists;
// *ok = false when this step's cell grid cannot use the fast neighbour
// search (a periodic side with fewer than three cells).
template <typename T>
mtd_status walk_desc(mtd_ctx *c, int n, const double *x, double *f, WalkDesc<T> &d, bool *ok) {
    if (!c->box_set) return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_box must be called before the first step");
    mtd_status st = ensure_capacity(c, n);
    if (st != MTD_OK) return st;
    const CellGrid g = make_grid(c);
    *ok = true;
    for (int a = 0; a < 3; ++a)
        if (g.periodic[a] && g.nc[a] < 3) *ok = false;
    if (!*ok) return MTD_OK;
    c->last_grid = g;
    if (c->plan_dirty) {
        build_plan(c);
        MTD_CU(cudaMemcpyAsync(c->d_plan, &c->plan, sizeof(BiasPlan), cudaMemcpyHostToDevice, c->st), "plan");
        MTD_CU(cudaStreamSynchronize(c->st), "plan");
        c->plan_dirty = false;
    }
    st = ensure_cells(c, g.ncell);
    if (st != MTD_OK) return st;
    SysDev s = sys_dev(c, x, nullptr, nullptr);
    s.count = c->count;
    s.start = c->start;
    Unit &u = c->units[0];
    Env &e = c->envs[u.env];
    std::memset(&d, 0, sizeof d);
    d.g = g;
    d.s = s;
    d.ns = neigh_spec(e);
    d.nd = env_dev(e);
    d.ld = local_dev<T>(c, u, g);
    d.f_src = f;
    d.f_dst = f;
    d.nb = (n + kBlock - 1) / kBlock;
    d.nchunk = (g.ncell + 255) / 256;
    d.d_out = c->d_out;
    d.d_status = c->d_status;
    d.d_nhills = c->d_nhills;
    use_slot(c, 0);
    d.h_out = c->h_out;
    d.h_status = c->h_status;
    d.h_nhills = c->h_nhills;
    c->last_sys = s;
    c->last_x = x;
    c->last_mask = nullptr;
    c->step_gen += 1;
    c->skin_last = false;
    return MTD_OK;
}
template mtd_status walk_desc<float>(mtd_ctx *, int, const double *, double *, WalkDesc<float> &, bool *);
template mtd_status walk_desc<double>(mtd_ctx *, int, const double *, double *, WalkDesc<double> &, bool *);

template void run_values<float>(mtd_ctx *, const CellGrid &, const double *, const int *);
template void run_values<double>(mtd_ctx *, const CellGrid &, const double *, const int *);
template void run_forces<float>(mtd_ctx *, const SysDev &, const CellGrid &, const double *, const int *,
                                const double *, double *, bool);
template void run_forces<double>(mtd_ctx *, const SysDev &, const CellGrid &, const double *, const int *,
                                 const double *, double *, bool);

}  // namespace ctx
}  // namespace mtd

extern "C" {

void mtd_options_default(mtd_options *o) {
    static const char *names[] = {"all"};
    static const int bits[] = {1};
    o->precision = MTD_PREC_MIXED;
    o->device = 0;
    o->boltz = 8.617343e-5;
    o->n_groups = 1;
    o->group_names = names;
    o->group_bits = bits;
    o->hills_path = nullptr;
    o->work_dir = nullptr;
}

int mtd_abi_version(void) { return MTD_ABI_VERSION; }

mtd_status mtd_parse_args(int narg, const char *const *arg, const mtd_options *opt, char *err, int errlen) {
    mtd_options def;
    mtd_options_default(&def);
    if (!opt) opt = &def;
    GroupTable groups;
    for (int i = 0; i < opt->n_groups; ++i) {
        groups.names.push_back(opt->group_names[i]);
        groups.bits.push_back(opt->group_bits[i]);
    }
    Config cfg;
    std::string e = parse_fix_args(narg, arg, groups, cfg);
    std::vector<std::string> names;
    for (auto &s : cfg.symbols) names.push_back(s.name);
    for (int d = 0; e.empty() && d < cfg.cv_dim; ++d) {
        std::vector<ExprInstr> code;
        e = compile_expr(cfg.dims[d].expr, names, code);
    }
    if (err && errlen > 0) {
        std::strncpy(err, e.c_str(), (size_t)errlen - 1);
        err[errlen - 1] = '\0';
    }
    return e.empty() ? MTD_OK : MTD_ERR_PARSE;
}

mtd_status mtd_eval_expression(const char *expr, int nsym, const char *const *names, const double *values,
                               double *value, double *grad) {
    if (!expr || nsym < 0 || nsym > kMaxSymbols || (nsym > 0 && (!names || !values)) || !value) return MTD_ERR_INVALID_ARG;
    std::vector<std::string> sym(names, names + nsym);
    std::vector<ExprInstr> code;
    if (!compile_expr(expr, sym, code).empty()) return MTD_ERR_PARSE;
    double g[kMaxSymbols];
    *value = eval_expr_host(code, values, nsym, g);
    if (grad)
        for (int k = 0; k < nsym; ++k) grad[k] = g[k];
    return MTD_OK;
}

mtd_status mtd_create(int narg, const char *const *arg, const mtd_options *opt, mtd_ctx **out) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    mtd_options def;
    mtd_options_default(&def);
    if (!opt) opt = &def;
    mtd_ctx *c = new mtd_ctx();
    c->fp64 = opt->precision == MTD_PREC_FP64;
    c->device = opt->device;
    c->boltz = opt->boltz;
    for (int i = 0; i < opt->n_groups; ++i) {
        c->groups.names.push_back(opt->group_names[i]);
        c->groups.bits.push_back(opt->group_bits[i]);
    }
    if (opt->hills_path) c->hills_path = opt->hills_path;
    if (opt->work_dir) c->work_dir = opt->work_dir;
    std::string e = parse_fix_args(narg, arg, c->groups, c->cfg);
    if (!e.empty()) {
        // a parse error leaves a context only to report the message
        c->err = e;
        *out = c;
        return MTD_ERR_PARSE;
    }
    for (auto &kv : c->cfg.cals)
        if (kv.second.kind == CAL_STRU_FACTOR_K && kv.second.nk > 1024) {
            c->err = "Error: STRU_FACTOR_K supports at most 1024 k-vectors.";
            *out = c;
            return MTD_ERR_UNSUPPORTED;
        }
    if (cudaSetDevice(c->device) != cudaSuccess) {
        c->err = "cudaSetDevice failed";
        *out = c;
        return MTD_ERR_CUDA;
    }
    cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
    c->own_st = c->st;
    cudaStreamCreateWithFlags(&c->side_st, cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&c->f_ready, cudaEventDisableTiming);
    c->cv.assign(c->cfg.cv_dim, 0.0);
    mtd_status s = plan_units(c);
    if (s == MTD_OK) {
        cudaError_t ce = cudaSuccess;
        ce = dalloc(&c->d_plan, sizeof(BiasPlan));
        if (ce == cudaSuccess) ce = dalloc(&c->d_out, sizeof(double) * 64);
        if (ce == cudaSuccess) ce = dalloc(&c->d_status, sizeof(DevStatus));
        if (ce == cudaSuccess) ce = dalloc(&c->d_hills, sizeof(HillRec) * kHillCap);
        if (ce == cudaSuccess) ce = dalloc(&c->d_nhills, sizeof(unsigned long long));
        if (ce == cudaSuccess) ce = dalloc(&c->d_vir, sizeof(double) * 8);
        if (ce == cudaSuccess) ce = cudaMemset(c->d_out, 0, sizeof(double) * 64);
        if (ce == cudaSuccess) ce = cudaMemset(c->d_status, 0, sizeof(DevStatus));
        if (ce == cudaSuccess) ce = cudaMemset(c->d_nhills, 0, sizeof(unsigned long long));
        if (ce == cudaSuccess) ce = cudaMallocHost((void **)&c->h_slots, sizeof(OutSlot) * kOutSlots);
        if (ce == cudaSuccess) {
            std::memset(c->h_slots, 0, sizeof(OutSlot) * kOutSlots);
            use_slot(c, 0);
        }
        for (int k = 0; k < kOutSlots && ce == cudaSuccess; ++k)
            ce = cudaEventCreateWithFlags(&c->slot_ev[k], cudaEventDisableTiming);
        s = cuda_check(c, ce, "context allocation");
    }
    *out = c;
    return s;
}

void mtd_destroy(mtd_ctx *c) {
    if (!c) return;
    if (c->st) cudaStreamSynchronize(c->st);
    if (c->h_slots) drain(c, true);   // hills of steps not yet collected still reach the HILLS file
    for (Env &e : c->envs) {
        dfree(e.list); dfree(e.count); dfree(e.key_r2); dfree(e.key_id); dfree(e.nkept);
        dfree(e.cand); dfree(e.ccount);
    }
    dfree(c->xref);
    dfree(c->d_skin);
    dfree(c->d_rbar);
    for (Unit &u : c->units) {
        void **arrs[] = {&u.q, &u.nf, &u.lq, &u.lqs, &u.e12, &u.lam, &u.g, &u.tu, &u.Q, &u.S, &u.w};
        for (void **a : arrs) dfree(*a);
        dfree(u.partials); dfree(u.coef); dfree(u.kvec); dfree(u.rho); dfree(u.skn); dfree(u.d_wtab);
    }
    dfree(c->d_x); dfree(c->d_fin); dfree(c->d_fout); dfree(c->d_mask); dfree(c->d_image);
    dfree(c->cellof); dfree(c->slot); dfree(c->perm); dfree(c->iperm); dfree(c->smask); dfree(c->arrival);
    dfree(c->xs); dfree(c->pf); dfree(c->count); dfree(c->start); dfree(c->d_vpart);
    dfree(c->d_plan); dfree(c->d_grid); dfree(c->d_hills); dfree(c->d_nhills); dfree(c->d_out);
    dfree(c->d_status); dfree(c->d_vir);
    if (c->h_slots) cudaFreeHost(c->h_slots);
    for (int k = 0; k < kOutSlots; ++k)
        if (c->slot_ev[k]) cudaEventDestroy(c->slot_ev[k]);
    if (c->own_st) cudaStreamDestroy(c->own_st);
    if (c->side_st) cudaStreamDestroy(c->side_st);
    if (c->nb) mtd_nnbias_destroy(c->nb);
    dfree(c->d_vdv);
    dfree(c->d_ws1);
    dfree(c->d_types);
    dfree(c->d_dcv);
    dfree(c->d_xchg);
    if (c->h_xchg) cudaFreeHost(c->h_xchg);
    if (c->f_ready) cudaEventDestroy(c->f_ready);
    if (c->prof_created)
        for (int i = 0; i < kProfMax; ++i) cudaEventDestroy(c->prof.ev[i]);
    if (c->f_hills) std::fclose(c->f_hills);
    if (c->f_rec) std::fclose(c->f_rec);
    delete c;
}

mtd_status mtd_set_box(mtd_ctx *c, const double lo[3], const double hi[3], const int periodic[3]) {
    if (!c || !lo || !hi || !periodic) return MTD_ERR_INVALID_ARG;
    for (int d = 0; d < 3; ++d) {
        if (!(hi[d] > lo[d])) return fail(c, MTD_ERR_INVALID_ARG, "box upper bound must exceed the lower bound");
        c->lo[d] = lo[d];
        c->hi[d] = hi[d];
        c->periodic[d] = periodic[d] ? 1 : 0;
    }
    double rmax = 0.0;
    for (const Env &e : c->envs) rmax = std::fmax(rmax, e.rc);
    for (int d = 0; d < 3; ++d)
        if (c->periodic[d] && hi[d] - lo[d] < 2.0 * rmax)
            return fail(c, MTD_ERR_INVALID_ARG, "Warning: box < cutoff_r, please check your system ! (periodic box must be >= 2 cutoff_r)");
    c->box_set = true;
    c->skin_valid = false;
    return MTD_OK;
}

mtd_status mtd_init(mtd_ctx *c) {
    if (!c) return MTD_ERR_INVALID_ARG;
    if (c->initialized) return MTD_OK;
    MTD_CU(dalloc(&c->d_ws1, sizeof(WalkState)), "bias state");
    MTD_CU(cudaMemset(c->d_ws1, 0, sizeof(WalkState)), "bias state");
    if (c->cfg.hill_list()) {   // hills kept as a list: exact FP64 sum and the learned bias
        double lo[kMaxDim], hi[kMaxDim];
        for (int d = 0; d < c->cfg.cv_dim; ++d) {
            lo[d] = c->cfg.dims[d].lo;
            hi[d] = c->cfg.dims[d].hi;
        }
        if (mtd_nnbias_create(c->cfg.cv_dim, lo, hi, 12345, &c->nb) != MTD_OK)
            return fail(c, MTD_ERR_CUDA, c->nb ? mtd_nnbias_last_error(c->nb) : "learned bias");
        MTD_CU(dalloc(&c->d_vdv, sizeof(double) * 8), "bias at s");
        c->grid_size = 0;
    } else {
        c->grid_size = 1;
        for (int d = 0; d < c->cfg.cv_dim; ++d) c->grid_size *= c->cfg.dims[d].nbins;
        MTD_CU(dalloc(&c->d_grid, sizeof(double) * (size_t)c->grid_size), "bias grid");
        MTD_CU(cudaMemset(c->d_grid, 0, sizeof(double) * (size_t)c->grid_size), "bias grid");
    }
    c->plan_dirty = true;
    build_plan(c);
    MTD_CU(cudaMemcpy(c->d_plan, &c->plan, sizeof(BiasPlan), cudaMemcpyHostToDevice), "plan");
    c->plan_dirty = false;
    const std::string hp = path_in(c, c->hills_path);
    bool appended = false;
    if (c->cfg.restart && !hp.empty()) {
        std::vector<HillRec> recs;
        bool exists = false;
        mtd_status s = read_hills(c, hp, recs, &exists);
        if (s != MTD_OK) return s;
        // an empty file counts as absent: it is rewritten with the header
        // (the reference restarts only from a file of non-zero size,
        // GH_t0_uniformGrid.cu:118, :175-181)
        if (exists) {
            FILE *f = std::fopen(hp.c_str(), "rb");
            long size = 0;
            if (f) {
                std::fseek(f, 0, SEEK_END);
                size = std::ftell(f);
                std::fclose(f);
            }
            exists = size > 0;
        }
        if (exists) {
            s = replay_records(c, recs);
            if (s != MTD_OK) return s;
            c->f_hills = std::fopen(hp.c_str(), "a");
            appended = true;
        }
    }
    if (c->dom_rank != 0) {   // domain decomposition: rank 0 alone writes HILLS and the record file
        if (c->f_hills) std::fclose(c->f_hills);
        c->f_hills = nullptr;
        c->initialized = true;
        return MTD_OK;
    }
    if (!hp.empty() && !appended) {
        c->f_hills = std::fopen(hp.c_str(), "w");
        if (!c->f_hills) return fail(c, MTD_ERR_IO, "Cannot open HILLS file for writing/appending.");
        if (c->cfg.cv_dim == 2) std::fprintf(c->f_hills, "# step cv1 cv2 height sigma\n");
        if (c->cfg.cv_dim == 1) std::fprintf(c->f_hills, "# step cv_values height sigma\n");
        std::fflush(c->f_hills);
    }
    if (!c->cfg.rec_file.empty()) {
        c->f_rec = std::fopen(path_in(c, c->cfg.rec_file).c_str(), "w+");
        if (c->f_rec) {
            std::fprintf(c->f_rec, "# step");
            for (int d = 0; d < c->cfg.cv_dim; ++d) std::fprintf(c->f_rec, " s%d", d + 1);
            std::fprintf(c->f_rec, " bias_energy\n");
            std::fflush(c->f_rec);
        }
    }
    c->initialized = true;
    return MTD_OK;
}

namespace {
// The part of mtd_post_force after x (and mask) are on the device: f upload
// beside the CV passes, the step with its overflow retries, f download.
mtd_status step_uploaded(mtd_ctx *c, int64_t step, int n, bool has_mask, const int *image, double *f,
                         double virial[6]) {
    const size_t b3 = sizeof(double) * 3 * (size_t)n;
    const int *mask = has_mask ? c->d_mask : nullptr;
    mtd_status s = MTD_OK;
    // f in pinned host memory, one STEINH L unit, no virial: the force pass
    // writes f over the host link in caller order (zero copy, no download),
    // and with mode 3 also reads it there (no upload)
    double *zf = nullptr;
    c->copy_used = 0;
    if (!virial && n >= 4096 && single_local_unit(c)) {
        cudaPointerAttributes pa{};
        if (cudaPointerGetAttributes(&pa, f) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer)
            zf = static_cast<double *>(pa.devicePointer);
        else
            cudaGetLastError();
    }
    // the mode: the caller's, else the one timing picked, else the next to try
    // (the first eligible call warms up in mode 3 and is not counted)
    int mode = c->host_copy_mode;
    if (mode == 0 && zf) {
        if (c->copy_pick) mode = c->copy_pick;
        else mode = c->copy_calls == 0 ? 3 : 1 + (c->copy_calls - 1) % 3;
        c->copy_used = mode;
    } else if (mode == 0) {
        mode = 3;
    }
    if (mode < 2) zf = nullptr;
    const bool upload = !zf || mode == 2;
    if (upload) {
        MTD_CU(cudaEventRecord(c->f_ready, c->st), "force upload");   // the side copies start after the previous step
        MTD_CU(cudaStreamWaitEvent(c->side_st, c->f_ready, 0), "force upload");
        MTD_CU(h2d_pieces(c->d_fin, f, b3, c->side_st), "f upload");
        if (image && virial)
            MTD_CU(cudaMemcpyAsync(c->d_image, image, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->side_st),
                   "image upload");
        MTD_CU(cudaEventRecord(c->f_ready, c->side_st), "force upload");
    }
    for (int attempt = 0; attempt < 4; ++attempt) {
        MTD_CU(cudaMemsetAsync(c->d_status, 0, sizeof(DevStatus), c->st), "status");
        c->zc_on = zf != nullptr;
        s = enqueue_step(c, step, n, c->d_x, mask, (image && virial) ? c->d_image : nullptr, upload ? c->d_fin : zf,
                         zf ? zf : c->d_fout, virial != nullptr, upload ? c->f_ready : nullptr);
        c->zc_on = false;
        if (s != MTD_OK) return s;
        // the forces go back in the same stream pass (a failed attempt's are
        // overwritten by the retry; with zero copy a failed attempt writes f back unchanged)
        if (!zf) MTD_CU(cudaMemcpyAsync(f, c->d_fout, b3, cudaMemcpyDeviceToHost, c->st), "f download");
        prof_mark("f_download", c->st);
        MTD_CU(cudaStreamSynchronize(c->st), "step");
        if (c->h_status->overflow == 0 && c->h_status->cand_overflow == 0) break;
        c->fifo.pop_back();   // the failed attempt is not collected
        // neighbour capacity too small: grow and run the step again
        s = grow_lists(c, c->h_status->overflow, c->h_status->cand_overflow);
        if (s != MTD_OK) return s;
        if (attempt == 3) return fail(c, MTD_ERR_NEIGH_OVERFLOW, "neighbour list capacity exceeded");
    }
    s = drain(c, true);
    if (s != MTD_OK) return s;
    if (virial)
        for (int t = 0; t < 6; ++t) virial[t] = c->virial[t];
    return MTD_OK;
}
}  // namespace

// Host copy mode 0: after the call, the wall time of a trial call counts for
// its mode; once each of modes 1-3 has three, the mode with the fastest call
// is kept (the minimum: a call slowed by something else says nothing about
// its mode, while the mean of three would carry it).
static void record_copy_trial(mtd_ctx *c, double ms) {
    if (c->copy_pick || c->copy_used == 0) return;
    const int m = c->copy_used;
    if (c->copy_calls > 0) {
        c->copy_ms[m] = c->copy_cnt[m] ? std::min(c->copy_ms[m], ms) : ms;
        c->copy_cnt[m] += 1;
    }
    c->copy_calls += 1;
    if (c->copy_cnt[1] >= 3 && c->copy_cnt[2] >= 3 && c->copy_cnt[3] >= 3) {
        int best = 3;
        for (int k = 1; k <= 3; ++k)
            if (c->copy_ms[k] < c->copy_ms[best]) best = k;
        c->copy_pick = best;
    }
}

mtd_status mtd_post_force(mtd_ctx *c, int64_t step, int n, const double *x, const int *mask, const int *image,
                          double *f, double virial[6]) {
    if (!c || n < 0 || (n > 0 && (!x || !f))) return MTD_ERR_INVALID_ARG;
    const auto t_call = std::chrono::steady_clock::now();
    if (!c->initialized) {
        mtd_status s = mtd_init(c);
        if (s != MTD_OK) return s;
    }
    mtd_status s = ensure_capacity(c, n);
    if (s != MTD_OK) return s;
    const size_t b3 = sizeof(double) * 3 * (size_t)n;
    // x (and mask) first on the step's stream; f (and image, read by the force
    // kernels only) on the side stream, overlapping the CV passes
    ProfScope prof_scope(c);
    MTD_CU(h2d_pieces(c->d_x, x, b3, c->st), "x upload");
    prof_mark("x_upload", c->st);
    if (mask) MTD_CU(cudaMemcpyAsync(c->d_mask, mask, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->st), "mask upload");
    s = step_uploaded(c, step, n, mask != nullptr, image, f, virial);
    if (s == MTD_OK)
        record_copy_trial(c, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_call).count());
    return s;
}

mtd_status mtd_set_positions_f64(mtd_ctx *c, const double *x, const int *type, const int *mask, int n, int groupbit) {
    if (!c || n < 0 || (n > 0 && !x)) return MTD_ERR_INVALID_ARG;
    if (groupbit == 0) return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_positions_f64: groupbit must be non-zero");
    if (!c->initialized) {
        mtd_status s = mtd_init(c);
        if (s != MTD_OK) return s;
    }
    mtd_status s = ensure_capacity(c, n);
    if (s != MTD_OK) return s;
    if (type && mtd_needs_types(c)) {
        s = mtd_set_types(c, n, type);
        if (s != MTD_OK) return s;
    }
    MTD_CU(h2d_pieces(c->d_x, x, sizeof(double) * 3 * (size_t)n, c->st), "x upload");
    if (mask) MTD_CU(cudaMemcpyAsync(c->d_mask, mask, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, c->st), "mask upload");
    MTD_CU(cudaStreamSynchronize(c->st), "x upload");   // the caller's arrays are borrowed for this call only
    c->staged_n = n;
    c->staged_mask = mask != nullptr;
    c->fix_groupbit = groupbit;
    return MTD_OK;
}

mtd_status mtd_step(mtd_ctx *c, int64_t step, double *f_inout, double *cv_out, double *bias_energy_out,
                    double virial_out[6]) {
    if (!c) return MTD_ERR_INVALID_ARG;
    if (c->staged_n < 0) return fail(c, MTD_ERR_INVALID_ARG, "mtd_step: call mtd_set_positions_f64 first");
    if (c->staged_n > 0 && !f_inout) return MTD_ERR_INVALID_ARG;
    const int n = c->staged_n;
    c->staged_n = -1;
    mtd_status s = ensure_capacity(c, n);
    if (s != MTD_OK) return s;
    s = step_uploaded(c, step, n, c->staged_mask, nullptr, f_inout, virial_out);
    if (s != MTD_OK) return s;
    if (cv_out)
        for (int d = 0; d < c->cfg.cv_dim; ++d) cv_out[d] = c->cv[d];
    if (bias_energy_out) *bias_energy_out = c->bias;
    return MTD_OK;
}

mtd_status mtd_create_from_config(const mtd_config *cfg, mtd_ctx **out) {
    if (!cfg || !out) return MTD_ERR_INVALID_ARG;
    return mtd_create(cfg->narg, cfg->arg, &cfg->opt, out);
}

mtd_status mtd_post_force_device(mtd_ctx *c, int64_t step, int n, const double *d_x, const int *d_mask,
                                 const int *d_image, const double *d_f_in, double *d_f_out) {
    if (!c || n < 0 || (n > 0 && (!d_x || !d_f_in || !d_f_out))) return MTD_ERR_INVALID_ARG;
    if (!c->initialized) {
        mtd_status s = mtd_init(c);
        if (s != MTD_OK) return s;
    }
    // steps already finished are collected without waiting; the host waits
    // only when every output slot is in flight, or for the hill-list bias,
    // whose new hills join the list on the host before the next step
    mtd_status s = drain(c, c->nb != nullptr);
    while (s == MTD_OK && (int)c->fifo.size() >= kOutSlots) {
        MTD_CU(cudaEventSynchronize(c->slot_ev[c->fifo.front().slot]), "step outputs");
        s = drain(c, false);
    }
    if (s != MTD_OK) return s;
    return enqueue_step(c, step, n, d_x, d_mask, d_image, d_f_in, d_f_out, false);
}

mtd_status mtd_sync(mtd_ctx *c) {
    if (!c) return MTD_ERR_INVALID_ARG;
    MTD_CU(cudaStreamSynchronize(c->st), "sync");
    const mtd_status sd = drain(c, true);
    if (sd != MTD_OK) return sd;
    if (c->overflow_seen || c->overflow_cand_seen) {
        const unsigned need = c->overflow_seen, cneed = c->overflow_cand_seen;
        c->overflow_seen = 0;
        c->overflow_cand_seen = 0;
        const mtd_status sg = grow_lists(c, need, cneed);
        if (sg != MTD_OK) return sg;
        cudaMemset(c->d_status, 0, sizeof(DevStatus));
        c->h_status->overflow = 0;
        c->h_status->cand_overflow = 0;
        c->pending = false;
        return fail(c, MTD_ERR_NEIGH_OVERFLOW, "neighbour list capacity exceeded; capacity grown, repeat the step");
    }
    return collect(c);
}

double mtd_compute_scalar(const mtd_ctx *c) { return c ? c->bias : 0.0; }

double mtd_compute_vector(const mtd_ctx *c, int k) {
    if (!c || k < 0 || k >= (int)c->cv.size()) return 0.0;
    return c->cv[k];
}

int mtd_cv_dim(const mtd_ctx *c) { return c ? c->cfg.cv_dim : 0; }

int mtd_last_launch_count(const mtd_ctx *c) { return c ? c->launches : 0; }

mtd_status mtd_set_stream(mtd_ctx *c, void *stream) {
    if (!c) return MTD_ERR_INVALID_ARG;
    MTD_CU(cudaStreamSynchronize(c->st), "stream switch");
    c->st = stream ? (cudaStream_t)stream : c->own_st;
    return MTD_OK;
}

mtd_status mtd_profile_enable(mtd_ctx *c, int enable) {
    if (!c) return MTD_ERR_INVALID_ARG;
    if (enable && !c->prof_created) {
        for (int i = 0; i < kProfMax; ++i) MTD_CU(cudaEventCreate(&c->prof.ev[i]), "profile events");
        c->prof_created = true;
    }
    if (c->prof.on) prof_collect(c);
    c->prof.on = enable != 0;
    c->prof.n = 0;
    c->prof_total.clear();
    return MTD_OK;
}

int mtd_profile_report(mtd_ctx *c, char *buf, int len) {
    if (!c) return 0;
    if (c->prof.on) prof_collect(c);
    std::string s;
    char line[160];
    for (auto &kv : c->prof_total) {
        std::snprintf(line, sizeof(line), "%s %lld %.6f\n", kv.first.c_str(), kv.second.first, kv.second.second);
        s += line;
    }
    if (buf && len > 0) {
        std::strncpy(buf, s.c_str(), (size_t)len - 1);
        buf[len - 1] = '\0';
    }
    return (int)s.size() + 1;
}

const char *mtd_last_error(const mtd_ctx *c) { return c ? c->err.c_str() : "null context"; }

}  // extern "C"
