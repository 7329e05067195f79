// walkers.cu -- multiple walkers sharing one bias grid (mtd_walkers_*).
#include "context.h"

// ------------------------------------------------------------------ multiple walkers
// W contexts built from the same `fix metad` arguments share walker 0's bias
// grid.  A step enqueues every walker's cell list, neighbour lists and CV
// values on its own stream, joins them for the three multi-walker bias
// kernels (WT heights from the grid at the start of the step, deposits in
// walker order, per-walker V, dV/ds and force coefficients), and forks again
// for the forces.  With the CUDA graph enabled the whole step is captured
// once per (atom counts, array pointers) and replayed; the step number
// travels through device memory.
//
// Decks whose walkers hold one STEINH L unit (one or two orders) on one
// neighbour environment, without skin lists and not sharded over ranks, run
// the step instead as ONE persistent kernel launch (walk_step.cu): the same
// bodies, the same block partials, the same results bit for bit.
struct mtd_walkers {
    std::vector<mtd_ctx *> w;
    std::string err;
    cudaStream_t st = nullptr;
    cudaEvent_t ev_start = nullptr, ev_bias = nullptr;
    std::vector<cudaEvent_t> ev_done;
    BiasPlan **d_plans = nullptr;
    WalkState *d_ws = nullptr;
    long long *d_step = nullptr, *h_step = nullptr;
    std::string hills_path = "HILLS";
    FILE *f_hills = nullptr;
    unsigned long long hills_written = 0;
    bool initialized = false;
    bool use_graph = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<int> g_n;
    std::vector<const double *> g_x;
    std::vector<double *> g_f;
    bool pending = false;
    long long pending_step = 0;
    int launches = 0;
    // sharded over ranks (mtd_walkers_set_ranks*): this object's walkers are
    // the global walkers rank * nwalk .. rank * nwalk + nwalk - 1
    int rank = 0, nranks = 0;                 // nranks 0: not sharded
    mtd_allgather_fn ag = nullptr;
    mtd_allgather_device_fn ag_dev = nullptr;
    void *ag_user = nullptr;
    double *d_xloc = nullptr, *d_xall = nullptr;   // [nwalk][kWalkRec], [nranks * nwalk][kWalkRec]
    double *h_xloc = nullptr, *h_xall = nullptr;   // pinned staging of the same
    // persistent single-launch step
    bool persist_enabled = true;              // mtd_walkers_enable_persistent
    bool persist_last = false;                // the last step ran as one launch
    void *d_desc = nullptr;                   // WalkDesc<T>[nwalk]
    std::vector<unsigned char> h_desc;        // the descriptors last uploaded
    int *d_pre = nullptr;                     // prefix sums: atom blocks, then cell chunks (2 (nwalk + 1))
    std::vector<int> h_pre;
    GridBar *d_bar = nullptr;
    int persist_blocks = 0;
    int wait_limit = 1 << 22;                 // barrier polls (mtd_walkers_set_wait)
    int wait_stall = 0;
};

namespace {

mtd_status wfail(mtd_walkers *W, mtd_status s, const std::string &m) {
    W->err = m;
    return s;
}

#define MTD_WCU(expr, what)                                                                          \
    do {                                                                                             \
        cudaError_t e_ = (expr);                                                                     \
        if (e_ != cudaSuccess) return wfail(W, MTD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void walkers_drop_graph(mtd_walkers *W) {
    if (W->gexec) cudaGraphExecDestroy(W->gexec);
    if (W->graph) cudaGraphDestroy(W->graph);
    W->gexec = nullptr;
    W->graph = nullptr;
}

// The step's work on the group stream and the walker streams.
mtd_status walkers_enqueue(mtd_walkers *W, long long step, const int *n, const double *const *d_x,
                           double *const *d_f) {
    const int nw = (int)W->w.size();
    PdlScope pdl_scope;   // each walker's kernel chain uses dependent launch (captured as programmatic edges)
    MTD_WCU(cudaMemcpyAsync(W->d_step, W->h_step, sizeof(long long), cudaMemcpyHostToDevice, W->st), "step");
    MTD_WCU(cudaEventRecord(W->ev_start, W->st), "fork");
    W->launches = 3;
    for (int k = 0; k < nw; ++k) {
        mtd_ctx *c = W->w[k];
        MTD_WCU(cudaStreamWaitEvent(c->st, W->ev_start, 0), "fork");
        c->launches = 0;
        mtd_status s = enqueue_values(c, n[k], d_x[k], nullptr, nullptr);
        if (s != MTD_OK) return wfail(W, s, "walker " + std::to_string(k) + ": " + c->err);
        MTD_WCU(cudaEventRecord(W->ev_done[k], c->st), "join");
        MTD_WCU(cudaStreamWaitEvent(W->st, W->ev_done[k], 0), "join");
    }
    if (W->nranks > 0) {   // this rank's hills out, every rank's hills in, all deposited in global order
        const int cnt = nw * kWalkRec, nall = W->nranks * nw;
        launch_walk_cvs_pack(W->d_plans, nw, W->d_step, W->d_ws, W->d_xloc, W->st);
        if (W->ag_dev) {
            if (W->ag_dev(W->d_xloc, cnt, W->d_xall, (void *)W->st, W->ag_user) != 0)
                return wfail(W, MTD_ERR_INVALID_ARG, "walker ranks: the device allgather callback failed");
            MTD_WCU(cudaGetLastError(), "walker allgather");
        } else {
            MTD_WCU(cudaMemcpyAsync(W->h_xloc, W->d_xloc, sizeof(double) * cnt, cudaMemcpyDeviceToHost, W->st), "hills out");
            MTD_WCU(cudaStreamSynchronize(W->st), "hills out");
            if (W->ag(W->h_xloc, cnt, W->h_xall, W->ag_user) != 0)
                return wfail(W, MTD_ERR_INVALID_ARG, "walker ranks: the allgather callback failed");
            MTD_WCU(cudaMemcpyAsync(W->d_xall, W->h_xall, sizeof(double) * nall * kWalkRec, cudaMemcpyHostToDevice,
                                    W->st), "hills in");
        }
        launch_walk_finish(W->d_plans, nw, W->d_step, W->d_ws, W->d_xall, nall, W->st);
        if (W->ag_dev)   // every rank's overflow flag, for mtd_walkers_sync
            MTD_WCU(cudaMemcpyAsync(W->h_xall, W->d_xall, sizeof(double) * nall * kWalkRec, cudaMemcpyDeviceToHost,
                                    W->st), "hills in");
        W->launches += 4;
    } else {
        launch_walk_bias(W->d_plans, nw, W->d_step, W->d_ws, W->st);
    }
    MTD_WCU(cudaGetLastError(), "walker bias");
    MTD_WCU(cudaEventRecord(W->ev_bias, W->st), "fork");
    for (int k = 0; k < nw; ++k) {
        mtd_ctx *c = W->w[k];
        MTD_WCU(cudaStreamWaitEvent(c->st, W->ev_bias, 0), "fork");
        mtd_status s = enqueue_forces(c, step, d_x[k], nullptr, d_f[k], d_f[k], false);
        if (s != MTD_OK) return wfail(W, s, "walker " + std::to_string(k) + ": " + c->err);
        W->launches += c->launches;
        MTD_WCU(cudaEventRecord(W->ev_done[k], c->st), "join");
        MTD_WCU(cudaStreamWaitEvent(W->st, W->ev_done[k], 0), "join");
    }
    return MTD_OK;
}

// The persistent path applies: every walker one STEINH L unit on one
// environment, no skin lists, not sharded, a step kernel for the orders.
bool persist_eligible(const mtd_walkers *W) {
    if (!W->persist_enabled || W->nranks > 0 || (int)W->w.size() > kWalkPersistMax) return false;
    for (const mtd_ctx *c : W->w)
        if (c->units.size() != 1 || c->units[0].kind != CAL_STEINH_L || c->envs.size() != 1 ||
            c->units[0].env != 0 || c->cfg.neigh_skin > 0.0)
            return false;
    return true;
}

template <typename T>
mtd_status walkers_persist_step(mtd_walkers *W, const int *n, const double *const *d_x, double *const *d_f,
                                bool *done) {
    const int nw = (int)W->w.size();
    *done = false;
    std::vector<unsigned char> desc(sizeof(WalkDesc<T>) * nw);
    std::vector<int> pre(2 * (nw + 1), 0);
    for (int k = 0; k < nw; ++k) {
        mtd_ctx *c = W->w[k];
        WalkDesc<T> d;
        bool ok = true;
        const mtd_status s = walk_desc<T>(c, n[k], d_x[k], d_f[k], d, &ok);
        if (s != MTD_OK) return wfail(W, s, "walker " + std::to_string(k) + ": " + c->err);
        if (!ok) return MTD_OK;   // a thin periodic box: the per-walker kernels handle it
        std::memcpy(desc.data() + sizeof(WalkDesc<T>) * k, &d, sizeof d);
        pre[k + 1] = pre[k] + d.nb;
        pre[nw + 1 + k + 1] = pre[nw + 1 + k] + d.nchunk;
    }
    const Unit &u = W->w[0]->units[0];
    const bool step_switch = u.sw_r.type == SW_STEP;
    if (!W->d_desc) {
        W->persist_blocks = walk_step_blocks<T>(u.LA, u.LB, step_switch);
        if (W->persist_blocks < 1) return MTD_OK;
        MTD_WCU(cudaMalloc(&W->d_desc, sizeof(WalkDesc<T>) * nw), "walker descriptors");
        MTD_WCU(cudaMalloc(&W->d_pre, sizeof(int) * 2 * (nw + 1)), "walker descriptors");
        MTD_WCU(cudaMalloc(&W->d_bar, sizeof(GridBar)), "grid barrier");
        MTD_WCU(cudaMemset(W->d_bar, 0, sizeof(GridBar)), "grid barrier");
    }
    const bool changed = desc != W->h_desc || pre != W->h_pre;
    if (changed) {   // new arguments: no graph holds the old ones
        walkers_drop_graph(W);
        MTD_WCU(cudaMemcpyAsync(W->d_desc, desc.data(), desc.size(), cudaMemcpyHostToDevice, W->st), "descriptors");
        MTD_WCU(cudaMemcpyAsync(W->d_pre, pre.data(), sizeof(int) * pre.size(), cudaMemcpyHostToDevice, W->st),
                "descriptors");
        MTD_WCU(cudaStreamSynchronize(W->st), "descriptors");
        W->h_desc.swap(desc);
        W->h_pre.swap(pre);
    }
    WalkStepArgs a{};
    a.nwalk = nw;
    a.pa = W->d_pre;
    a.pc = W->d_pre + nw + 1;
    a.plans = W->d_plans;
    a.step = W->h_step;   // pinned: the launch reads the step the host set
    a.ws = W->d_ws;
    a.bar = W->d_bar;
    a.limit = W->wait_limit;
    a.stall = W->wait_stall;
    const WalkDesc<T> *dd = static_cast<const WalkDesc<T> *>(W->d_desc);
    auto launch = [&]() {
        return launch_walk_step<T>(u.LA, u.LB, step_switch, dd, a, W->persist_blocks, W->st);
    };
    if (W->use_graph && !changed && W->gexec) {
        MTD_WCU(cudaGraphLaunch(W->gexec, W->st), "graph launch");
    } else if (W->use_graph && !changed) {
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamBeginCapture(W->st, cudaStreamCaptureModeThreadLocal);
        if (ce == cudaSuccess) {
            const cudaError_t le = launch();
            ce = cudaStreamEndCapture(W->st, &g);
            if (le != cudaSuccess) ce = le;
        }
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&W->gexec, g, 0);
        if (ce == cudaSuccess) {
            W->graph = g;
            MTD_WCU(cudaGraphLaunch(W->gexec, W->st), "graph launch");
        } else {   // the launch cannot be captured here: plain launches
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            W->gexec = nullptr;
            W->use_graph = false;
            MTD_WCU(launch(), "walker step launch");
        }
    } else {
        MTD_WCU(launch(), "walker step launch");
    }
    W->launches = 1;
    *done = true;
    return MTD_OK;
}

}  // namespace

extern "C" {

mtd_status mtd_walkers_create(int nwalk, int narg, const char *const *arg, const mtd_options *opt,
                              mtd_walkers **out) {
    if (!out) return MTD_ERR_INVALID_ARG;
    *out = nullptr;
    mtd_walkers *W = new mtd_walkers();
    *out = W;
    if (nwalk < 1 || nwalk > 1024) return wfail(W, MTD_ERR_INVALID_ARG, "nwalk must be in [1, 1024]");
    mtd_options o;
    mtd_options_default(&o);
    if (opt) o = *opt;
    if (o.hills_path) W->hills_path = o.hills_path;
    const std::string wd = o.work_dir ? o.work_dir : "";
    if (!W->hills_path.empty() && W->hills_path[0] != '/' && !wd.empty()) W->hills_path = wd + "/" + W->hills_path;
    o.hills_path = "";   // the group writes one HILLS file
    for (int k = 0; k < nwalk; ++k) {
        mtd_ctx *c = nullptr;
        const mtd_status s = mtd_create(narg, arg, &o, &c);
        if (c) c->ring = false;
        W->w.push_back(c);
        if (s != MTD_OK) return wfail(W, s, c ? c->err : "context creation failed");
        if (c->cfg.hill_list()) return wfail(W, MTD_ERR_UNSUPPORTED, "walkers share a grid: CV_dim <= 3, no NN_BIAS");
        if (k > 0) c->cfg.rec_file.clear();   // one RECORD file (walker 0's)
    }
    MTD_WCU(cudaStreamCreateWithFlags(&W->st, cudaStreamNonBlocking), "stream");
    MTD_WCU(cudaEventCreateWithFlags(&W->ev_start, cudaEventDisableTiming), "event");
    MTD_WCU(cudaEventCreateWithFlags(&W->ev_bias, cudaEventDisableTiming), "event");
    W->ev_done.resize(nwalk);
    for (int k = 0; k < nwalk; ++k)
        MTD_WCU(cudaEventCreateWithFlags(&W->ev_done[k], cudaEventDisableTiming), "event");
    MTD_WCU(cudaMalloc(&W->d_plans, sizeof(BiasPlan *) * nwalk), "plans");
    MTD_WCU(cudaMalloc(&W->d_ws, sizeof(WalkState) * nwalk), "walker state");
    MTD_WCU(cudaMemset(W->d_ws, 0, sizeof(WalkState) * nwalk), "walker state");
    MTD_WCU(cudaMalloc(&W->d_step, sizeof(long long)), "step");
    MTD_WCU(cudaMallocHost(&W->h_step, sizeof(long long)), "step");
    return MTD_OK;
}

void mtd_walkers_destroy(mtd_walkers *W) {
    if (!W) return;
    if (W->st) cudaStreamSynchronize(W->st);
    walkers_drop_graph(W);
    for (size_t k = 0; k < W->w.size(); ++k) {
        if (!W->w[k]) continue;
        if (k > 0 && W->initialized) W->w[k]->d_grid = nullptr;   // walker 0 owns the shared grid
        mtd_destroy(W->w[k]);
    }
    for (cudaEvent_t e : W->ev_done)
        if (e) cudaEventDestroy(e);
    if (W->ev_start) cudaEventDestroy(W->ev_start);
    if (W->ev_bias) cudaEventDestroy(W->ev_bias);
    if (W->d_plans) cudaFree(W->d_plans);
    if (W->d_ws) cudaFree(W->d_ws);
    if (W->d_step) cudaFree(W->d_step);
    if (W->h_step) cudaFreeHost(W->h_step);
    if (W->d_xloc) cudaFree(W->d_xloc);
    if (W->d_xall) cudaFree(W->d_xall);
    if (W->h_xloc) cudaFreeHost(W->h_xloc);
    if (W->h_xall) cudaFreeHost(W->h_xall);
    if (W->d_desc) cudaFree(W->d_desc);
    if (W->d_pre) cudaFree(W->d_pre);
    if (W->d_bar) cudaFree(W->d_bar);
    if (W->st) cudaStreamDestroy(W->st);
    if (W->f_hills) std::fclose(W->f_hills);
    delete W;
}

const char *mtd_walkers_last_error(const mtd_walkers *W) { return W ? W->err.c_str() : "null object"; }

int mtd_walkers_count(const mtd_walkers *W) { return W ? (int)W->w.size() : 0; }

mtd_status mtd_walkers_set_box(mtd_walkers *W, int k, const double lo[3], const double hi[3],
                               const int periodic[3]) {
    if (!W || k < 0 || k >= (int)W->w.size()) return MTD_ERR_INVALID_ARG;
    walkers_drop_graph(W);
    const mtd_status s = mtd_set_box(W->w[k], lo, hi, periodic);
    return s == MTD_OK ? s : wfail(W, s, W->w[k]->err);
}

mtd_status mtd_walkers_init(mtd_walkers *W) {
    if (!W) return MTD_ERR_INVALID_ARG;
    if (W->initialized) return MTD_OK;
    const int nw = (int)W->w.size();
    for (int k = 0; k < nw; ++k) {
        const mtd_status s = mtd_init(W->w[k]);
        if (s != MTD_OK) return wfail(W, s, W->w[k]->err);
    }
    mtd_ctx *c0 = W->w[0];
    std::vector<BiasPlan *> plans(nw);
    for (int k = 0; k < nw; ++k) {
        mtd_ctx *c = W->w[k];
        if (k > 0) {
            cudaFree(c->d_grid);
            c->d_grid = c0->d_grid;   // one grid for the group
        }
        build_plan(c);
        MTD_WCU(cudaMemcpy(c->d_plan, &c->plan, sizeof(BiasPlan), cudaMemcpyHostToDevice), "plan");
        c->plan_dirty = false;
        plans[k] = c->d_plan;
    }
    W->initialized = true;
    MTD_WCU(cudaMemcpy(W->d_plans, plans.data(), sizeof(BiasPlan *) * nw, cudaMemcpyHostToDevice), "plans");
    if (W->nranks > 0) {
        const size_t loc = sizeof(double) * nw * kWalkRec, all = loc * W->nranks;
        MTD_WCU(cudaMalloc((void **)&W->d_xloc, loc), "walker ranks");
        MTD_WCU(cudaMalloc((void **)&W->d_xall, all), "walker ranks");
        MTD_WCU(cudaHostAlloc((void **)&W->h_xloc, loc, cudaHostAllocDefault), "walker ranks");
        MTD_WCU(cudaHostAlloc((void **)&W->h_xall, all, cudaHostAllocDefault), "walker ranks");
        std::memset(W->h_xall, 0, all);
    }
    if (!W->hills_path.empty() && W->rank == 0) {   // sharded: rank 0 alone writes the group's HILLS
        W->f_hills = std::fopen(W->hills_path.c_str(), "w");
        if (!W->f_hills) return wfail(W, MTD_ERR_IO, "Cannot open HILLS file for writing/appending.");
        if (c0->cfg.cv_dim == 2) std::fprintf(W->f_hills, "# step cv1 cv2 height sigma\n");
        if (c0->cfg.cv_dim == 1) std::fprintf(W->f_hills, "# step cv_values height sigma\n");
        std::fflush(W->f_hills);
    }
    return MTD_OK;
}

static mtd_status walkers_set_ranks(mtd_walkers *W, int rank, int nranks, mtd_allgather_fn fn,
                             mtd_allgather_device_fn fn_dev, void *user) {
    if (!W) return MTD_ERR_INVALID_ARG;
    if (W->initialized) return wfail(W, MTD_ERR_INVALID_ARG, "walker ranks must be set before the first step");
    if (nranks < 1 || rank < 0 || rank >= nranks || (!fn && !fn_dev))
        return wfail(W, MTD_ERR_INVALID_ARG, "walker ranks need 0 <= rank < nranks and an allgather callback");
    W->rank = rank;
    W->nranks = nranks;
    W->ag = fn;
    W->ag_dev = fn_dev;
    W->ag_user = user;
    W->use_graph = false;   // the exchange sits between the captured phases
    return MTD_OK;
}

mtd_status mtd_walkers_set_ranks(mtd_walkers *W, int rank, int nranks, mtd_allgather_fn fn, void *user) {
    return walkers_set_ranks(W, rank, nranks, fn, nullptr, user);
}

mtd_status mtd_walkers_set_ranks_device(mtd_walkers *W, int rank, int nranks, mtd_allgather_device_fn fn,
                                        void *user) {
    return walkers_set_ranks(W, rank, nranks, nullptr, fn, user);
}

mtd_status mtd_walkers_enable_graph(mtd_walkers *W, int enable) {
    if (!W) return MTD_ERR_INVALID_ARG;
    if (W->st) cudaStreamSynchronize(W->st);
    walkers_drop_graph(W);
    W->use_graph = enable != 0 && W->nranks == 0;
    return MTD_OK;
}

mtd_status mtd_walkers_sync(mtd_walkers *W);

mtd_status mtd_walkers_step_device(mtd_walkers *W, int64_t step, const int *n, const double *const *d_x,
                                   double *const *d_f) {
    if (!W || !n || !d_x || !d_f) return MTD_ERR_INVALID_ARG;
    if (!W->initialized) {
        const mtd_status s = mtd_walkers_init(W);
        if (s != MTD_OK) return s;
    }
    const int nw = (int)W->w.size();
    for (int k = 0; k < nw; ++k)
        if (n[k] < 1 || !d_x[k] || !d_f[k]) return wfail(W, MTD_ERR_INVALID_ARG, "every walker needs atoms");
    if (W->pending) {
        const mtd_status s = mtd_walkers_sync(W);
        if (s != MTD_OK) return s;
    }
    *W->h_step = step;
    if (persist_eligible(W)) {
        bool done = false;
        const mtd_status s = W->w[0]->fp64 ? walkers_persist_step<double>(W, n, d_x, d_f, &done)
                                           : walkers_persist_step<float>(W, n, d_x, d_f, &done);
        if (s != MTD_OK) return s;
        if (done) {
            W->persist_last = true;
            W->g_n.clear();   // the per-walker graph (if any) no longer matches
            for (mtd_ctx *c : W->w) {
                c->pending = true;
                c->pending_step = step;
                c->want_virial = false;
            }
            W->pending = true;
            W->pending_step = step;
            return MTD_OK;
        }
    }
    W->persist_last = false;
    bool same = (int)W->g_n.size() == nw;
    for (int k = 0; same && k < nw; ++k) same = W->g_n[k] == n[k] && W->g_x[k] == d_x[k] && W->g_f[k] == d_f[k];
    if (W->use_graph && same && W->gexec) {
        MTD_WCU(cudaGraphLaunch(W->gexec, W->st), "graph launch");
    } else if (W->use_graph && same) {
        // the same arguments ran once eagerly (allocations done): capture, then launch
        MTD_WCU(cudaStreamBeginCapture(W->st, cudaStreamCaptureModeThreadLocal), "capture");
        const mtd_status s = walkers_enqueue(W, step, n, d_x, d_f);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(W->st, &g);
        if (s != MTD_OK) {
            if (g) cudaGraphDestroy(g);
            return s;
        }
        MTD_WCU(ce, "capture");
        W->graph = g;
        MTD_WCU(cudaGraphInstantiate(&W->gexec, W->graph, 0), "graph instantiate");
        MTD_WCU(cudaGraphLaunch(W->gexec, W->st), "graph launch");
    } else {
        walkers_drop_graph(W);
        W->g_n.assign(n, n + nw);
        W->g_x.assign(d_x, d_x + nw);
        W->g_f.assign(d_f, d_f + nw);
        const mtd_status s = walkers_enqueue(W, step, n, d_x, d_f);
        if (s != MTD_OK) return s;
    }
    for (mtd_ctx *c : W->w) {
        c->pending = true;
        c->pending_step = step;
        c->want_virial = false;
    }
    W->pending = true;
    W->pending_step = step;
    return MTD_OK;
}

mtd_status mtd_walkers_autotune(mtd_walkers *W, const int *n, const double *const *d_x, int reps, int *choices) {
    if (!W || !n || !d_x || reps < 1) return MTD_ERR_INVALID_ARG;
    if (!W->initialized) {
        const mtd_status s = mtd_walkers_init(W);
        if (s != MTD_OK) return s;
    }
    if (W->pending) {
        const mtd_status s = mtd_walkers_sync(W);
        if (s != MTD_OK) return s;
    }
    for (size_t k = 0; k < W->w.size(); ++k) {
        if (n[k] < 1 || !d_x[k]) return wfail(W, MTD_ERR_INVALID_ARG, "every walker needs atoms");
        const mtd_status s = autotune_idle(W->w[k], n[k], d_x[k], nullptr, reps, choices ? choices + 3 * k : nullptr);
        if (s != MTD_OK) return wfail(W, s, W->w[k]->err);
    }
    walkers_drop_graph(W);   // the next steps run (and capture) the chosen shapes
    W->g_n.clear();
    return MTD_OK;
}

mtd_status mtd_walkers_sync(mtd_walkers *W) {
    if (!W) return MTD_ERR_INVALID_ARG;
    MTD_WCU(cudaStreamSynchronize(W->st), "sync");
    if (!W->pending) return MTD_OK;
    W->pending = false;
    if (W->persist_last && W->d_bar) {   // a grid-barrier wait of the persistent step ran out
        GridBar hb{};
        MTD_WCU(cudaMemcpy(&hb, W->d_bar, sizeof hb, cudaMemcpyDeviceToHost), "grid barrier");
        if (hb.err) {
            MTD_WCU(cudaMemset(W->d_bar, 0, sizeof(GridBar)), "grid barrier");
            // the launch may have binned atoms without reaching the scatter
            // pass that zeroes the cell counts: zero them for the next build
            for (mtd_ctx *c : W->w)
                if (c->count) MTD_WCU(cudaMemset(c->count, 0, sizeof(int) * (size_t)c->cap_cell), "cell counts");
            MTD_WCU(cudaDeviceSynchronize(), "grid barrier");
            walkers_drop_graph(W);
            for (mtd_ctx *c : W->w) c->pending = false;
            return wfail(W, MTD_ERR_TIMEOUT,
                         "walker step: a grid-barrier wait ran out; the step is incomplete, repeat it");
        }
    }
    bool overflow = false;
    for (mtd_ctx *c : W->w) {
        if (c->h_status->overflow || c->h_status->cand_overflow) {
            const mtd_status s = grow_lists(c, c->h_status->overflow, c->h_status->cand_overflow);
            if (s != MTD_OK) return wfail(W, s, c->err);
            cudaMemset(c->d_status, 0, sizeof(DevStatus));
            c->h_status->overflow = 0;
            c->h_status->cand_overflow = 0;
            overflow = true;
        }
    }
    if (W->nranks > 0)   // sharded: a walker of any rank overflowed, so every rank repeats the step
        for (int r = 0; r < W->nranks * (int)W->w.size(); ++r)
            if (W->h_xall[(size_t)r * kWalkRec + kMaxDim + 2] != 0.0) overflow = true;
    if (overflow) {
        walkers_drop_graph(W);
        W->g_n.clear();
        for (mtd_ctx *c : W->w) c->pending = false;
        return wfail(W, MTD_ERR_NEIGH_OVERFLOW, "neighbour list capacity exceeded; capacity grown, repeat the step");
    }
    // the group's hills (walker 0's ring) go to the group HILLS file
    mtd_ctx *c0 = W->w[0];
    const unsigned long long nh = *c0->h_nhills;
    if (nh > W->hills_written) {
        unsigned long long from = W->hills_written;
        if (nh - from > (unsigned long long)kHillCap) from = nh - kHillCap;
        if (W->f_hills) {   // the new records in at most two copies (the ring wraps once at most)
            std::vector<HillRec> recs((size_t)(nh - from));
            const size_t a = (size_t)(from % kHillCap);
            const size_t first = std::min(recs.size(), (size_t)kHillCap - a);
            MTD_WCU(cudaMemcpy(recs.data(), c0->d_hills + a, sizeof(HillRec) * first, cudaMemcpyDeviceToHost),
                    "hills");
            if (first < recs.size())
                MTD_WCU(cudaMemcpy(recs.data() + first, c0->d_hills, sizeof(HillRec) * (recs.size() - first),
                                   cudaMemcpyDeviceToHost),
                        "hills");
            for (const HillRec &r : recs) {
                std::fprintf(W->f_hills, "%lld", r.step);
                for (int d = 0; d < c0->cfg.cv_dim; ++d) std::fprintf(W->f_hills, " %.16g", r.s[d]);
                std::fprintf(W->f_hills, " %.16g %.16g\n", r.w, r.sigma);
            }
            std::fflush(W->f_hills);
        }
        W->hills_written = nh;
    }
    for (mtd_ctx *c : W->w) {
        c->hills_written = nh;
        const mtd_status s = collect(c);
        if (s != MTD_OK) return wfail(W, s, c->err);
    }
    return MTD_OK;
}

double mtd_walkers_cv(const mtd_walkers *W, int k, int d) {
    if (!W || k < 0 || k >= (int)W->w.size()) return 0.0;
    return mtd_compute_vector(W->w[k], d);
}

double mtd_walkers_bias(const mtd_walkers *W, int k) {
    if (!W || k < 0 || k >= (int)W->w.size()) return 0.0;
    return mtd_compute_scalar(W->w[k]);
}

mtd_status mtd_walkers_get_grid(mtd_walkers *W, double *out, int64_t count) {
    if (!W || !out) return MTD_ERR_INVALID_ARG;
    MTD_WCU(cudaStreamSynchronize(W->st), "grid");
    const mtd_status s = mtd_get_grid(W->w[0], out, count);
    return s == MTD_OK ? s : wfail(W, s, W->w[0]->err);
}

int mtd_walkers_last_launch_count(const mtd_walkers *W) { return W ? W->launches : 0; }

mtd_status mtd_walkers_enable_persistent(mtd_walkers *W, int enable) {
    if (!W) return MTD_ERR_INVALID_ARG;
    if (W->st) cudaStreamSynchronize(W->st);
    walkers_drop_graph(W);
    W->g_n.clear();
    W->h_desc.clear();
    W->persist_enabled = enable != 0;
    return MTD_OK;
}

int mtd_walkers_persistent_active(const mtd_walkers *W) { return W && W->persist_last ? 1 : 0; }

mtd_status mtd_walkers_set_wait(mtd_walkers *W, int limit, int stall) {
    if (!W || limit < 0) return MTD_ERR_INVALID_ARG;
    if (W->st) cudaStreamSynchronize(W->st);
    walkers_drop_graph(W);
    W->h_desc.clear();
    W->wait_limit = limit > 0 ? limit : (1 << 22);
    W->wait_stall = stall ? 1 : 0;
    return MTD_OK;
}

}  // extern "C"
