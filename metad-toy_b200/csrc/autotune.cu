// autotune.cu -- the kernel-shape autotuner: times the interchangeable
// launch shapes of the kernels without block-level reductions on the caller's
// positions and keeps the fastest per context.  Every shape gives bitwise-
// identical results.  The reference has fixed launch shapes.
#include "context.h"

namespace mtd {
namespace ctx {

// The tuning passes of one idle context: a values pass on the given
// positions (lists grown until they fit), then each interchangeable kernel
// shape timed over `reps` launches with CUDA events on the context stream,
// the fastest kept.  The passes write only scratch (lists, per-atom records,
// d_fout); no step is recorded, no hill deposited.
mtd_status autotune_idle(mtd_ctx *c, int n, const double *d_x, const int *d_mask, int reps, int *choice) {
    const bool prof = c->prof.on;
    c->prof.on = false;
    mtd_status s = MTD_OK;
    for (int attempt = 0;; ++attempt) {
        MTD_CU(cudaMemsetAsync(c->d_status, 0, sizeof(DevStatus), c->st), "status");
        s = enqueue_values(c, n, d_x, d_mask, nullptr);
        if (s != MTD_OK) break;
        DevStatus hs{};
        MTD_CU(cudaMemcpyAsync(&hs, c->d_status, sizeof(DevStatus), cudaMemcpyDeviceToHost, c->st), "status");
        MTD_CU(cudaStreamSynchronize(c->st), "autotune");
        if (hs.overflow == 0 && hs.cand_overflow == 0) break;
        if (attempt == 3) {
            s = fail(c, MTD_ERR_NEIGH_OVERFLOW, "neighbour list capacity exceeded");
            break;
        }
        s = grow_lists(c, hs.overflow, hs.cand_overflow);
        if (s != MTD_OK) break;
    }
    if (s != MTD_OK) {
        c->prof.on = prof;
        return s;
    }
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MTD_CU(cudaEventCreate(&e0), "autotune");
    MTD_CU(cudaEventCreate(&e1), "autotune");
    auto timed = [&](auto &&fn) {
        fn();
        cudaEventRecord(e0, c->st);
        for (int r = 0; r < reps; ++r) fn();
        cudaEventRecord(e1, c->st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms;
    };
    const CellGrid g = c->last_grid;
    SysDev sd = c->last_sys;
    sd.skin = nullptr;   // the timed neighbour searches run in full (no skin gate)
    float best = 1e30f;
    for (int v = 0; v < 3; ++v) {
        const float t = timed([&] {
            for (Env &e : c->envs) {
                NeighSpec ns = neigh_spec(e);
                ns.variant = v;
                launch_neighbors(g, sd, ns, env_dev(e), c->d_status, c->st);
            }
        });
        if (t < best) {
            best = t;
            c->tune_nbr = v;
        }
    }
    const int shapes[2] = {256, 128};
    best = 1e30f;
    int bq = 256, bs = 0;
    for (int split = 0; split < (c->skin_last ? 2 : 1); ++split)
        for (int qb : shapes) {
            c->tune_q = qb;
            c->tune_qsplit = split;
            const float t = timed([&] {
                if (c->fp64) run_values<double>(c, g, d_x, d_mask);
                else run_values<float>(c, g, d_x, d_mask);
            });
            if (t < best) {
                best = t;
                bq = qb;
                bs = split;
            }
        }
    c->tune_q = bq;
    c->tune_qsplit = bs;
    best = 1e30f;
    int bl = 256;
    for (int lb : shapes) {
        c->tune_l = lb;
        const float t = timed([&] {
            if (c->fp64) run_forces<double>(c, sd, g, d_x, d_mask, c->d_fin, c->d_fout, false);
            else run_forces<float>(c, sd, g, d_x, d_mask, c->d_fin, c->d_fout, false);
        });
        if (t < best) {
            best = t;
            bl = lb;
        }
    }
    c->tune_l = bl;
    // S(k) shapes: k-vectors per pass of the value pass, unroll depth of the force pass
    for (Unit &u : c->units) {
        if (u.kind != CAL_STRU_FACTOR_K) continue;
        best = 1e30f;
        int bv = c->tune_skq;
        for (int qv : {4, 8, 16}) {
            c->tune_skq = qv;
            const float t = timed([&] {
                if (c->fp64) run_values<double>(c, g, d_x, d_mask);
                else run_values<float>(c, g, d_x, d_mask);
            });
            if (t < best) {
                best = t;
                bv = qv;
            }
        }
        c->tune_skq = bv;
        best = 1e30f;
        int bf = c->tune_skqf;
        for (int qf : {1, 2, 4}) {
            c->tune_skqf = qf;
            const float t = timed([&] {
                if (c->fp64) run_forces<double>(c, sd, g, d_x, d_mask, c->d_fin, c->d_fout, false);
                else run_forces<float>(c, sd, g, d_x, d_mask, c->d_fin, c->d_fout, false);
            });
            if (t < best) {
                best = t;
                bf = qf;
            }
        }
        c->tune_skqf = bf;
        break;   // one set of shapes per context
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    MTD_CU(cudaMemsetAsync(c->d_status, 0, sizeof(DevStatus), c->st), "status");
    MTD_CU(cudaStreamSynchronize(c->st), "autotune");
    c->prof.on = prof;
    if (choice) {
        choice[0] = c->tune_nbr;
        choice[1] = c->tune_q;
        choice[2] = c->tune_l;
    }
    return MTD_OK;
}

}  // namespace ctx
}  // namespace mtd

extern "C" {

mtd_status mtd_autotune(mtd_ctx *c, int n, const double *d_x, const int *d_mask, int reps, int choice[3]) {
    if (!c || n < 1 || !d_x || reps < 1) return MTD_ERR_INVALID_ARG;
    if (!c->initialized) {
        const mtd_status s = mtd_init(c);
        if (s != MTD_OK) return s;
    }
    if (!c->box_set) return fail(c, MTD_ERR_INVALID_ARG, "mtd_set_box must be called before mtd_autotune");
    const mtd_status s = mtd_sync(c);
    if (s != MTD_OK) return s;
    return autotune_idle(c, n, d_x, d_mask, reps, choice);
}

mtd_status mtd_get_tuning(mtd_ctx *c, int out[6]) {
    if (!c || !out) return MTD_ERR_INVALID_ARG;
    out[0] = c->tune_nbr;
    out[1] = c->tune_q;
    out[2] = c->tune_l;
    out[3] = c->tune_qsplit;
    out[4] = c->tune_skq;
    out[5] = c->tune_skqf;
    return MTD_OK;
}

mtd_status mtd_set_tuning_all(mtd_ctx *c, const int in[6]) {
    if (!c || !in) return MTD_ERR_INVALID_ARG;
    mtd_status s = mtd_set_tuning(c, in[0], in[1], in[2]);
    if (s != MTD_OK) return s;
    if (in[3] != 0 && in[3] != 1) return MTD_ERR_INVALID_ARG;
    s = mtd_set_sk_tiles(c, in[4], in[5]);
    if (s != MTD_OK) return s;
    c->tune_qsplit = in[3];
    return MTD_OK;
}

mtd_status mtd_sk_tiles(mtd_ctx *c, int *q_values, int *q_force) {
    if (!c) return MTD_ERR_INVALID_ARG;
    if (q_values) *q_values = c->tune_skq;
    if (q_force) *q_force = c->tune_skqf;
    return MTD_OK;
}

mtd_status mtd_set_sk_tiles(mtd_ctx *c, int q_values, int q_force) {
    if (!c || (q_values != 4 && q_values != 8 && q_values != 16) || (q_force != 1 && q_force != 2 && q_force != 4))
        return MTD_ERR_INVALID_ARG;
    c->tune_skq = q_values;
    c->tune_skqf = q_force;
    return MTD_OK;
}

mtd_status mtd_set_tuning(mtd_ctx *c, int neighbor_shape, int q_block, int lambda_block) {
    if (!c || neighbor_shape < 0 || neighbor_shape > 2) return MTD_ERR_INVALID_ARG;
    if ((q_block != 0 && q_block != 128 && q_block != 256) || (lambda_block != 0 && lambda_block != 128 &&
                                                               lambda_block != 256))
        return MTD_ERR_INVALID_ARG;
    c->tune_nbr = neighbor_shape;
    c->tune_q = q_block;
    c->tune_l = lambda_block;
    return MTD_OK;
}

}  // extern "C"
