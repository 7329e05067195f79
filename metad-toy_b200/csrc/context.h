// context.h -- internal to libmetad_b200.so: the context object behind the C
// ABI and the helpers shared by the files that implement it:
//   context.cu   set-up, the per-step launch sequence, output collection
//   decomp.cu    domain decomposition: the per-step exchange of unit totals
//   hills.cu     HILLS file, restart replay, hill-list bias bookkeeping
//   autotune.cu  kernel-shape autotuner
//   peratom.cu   per-atom exports (compute metad/atom), atom types, neighbour lists
//   walkers.cu   multiple walkers sharing one grid
#pragma once

#include "../../include/metad_b200.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <string>
#include <vector>

#include "args.h"
#include "expr.h"
#include "kernels.h"
#include "nnbias.h"

namespace mtd {
namespace ctx {

enum EnvKind { ENV_Q = 0, ENV_L = 1, ENV_R = 2 };

struct Env {
    int kind = ENV_R;
    double rc = 0;
    int cap = 0;
    SwParams sw{};
    double eps = 0;
    int M = 0;
    int cap_n = 0;
    int *list = nullptr;
    int *count = nullptr;
    double *key_r2 = nullptr;
    int *key_id = nullptr;
    int *nkept = nullptr;
    std::vector<int> cals;
    // skin lists (NEIGH_SKIN): candidates within cutoff + skin, slot-major [Mc][npad]
    int Mc = 0;
    int *cand = nullptr;
    int *ccount = nullptr;
};

struct Unit {
    int kind = 0;                 // CalKind
    std::vector<std::string> calnames;
    int env = -1;
    int LA = 0, LB = 0;
    int groupbit = 1;
    SwParams sw_r{}, sw_cvA{}, sw_cvB{};
    std::vector<SwParams> qsw;
    std::vector<std::string> qswnames;
    double rc = 0, qf = 0;
    SwParams sf_sw{};
    bool dsig = false;
    bool used = false;
    int cap_n = 0;
    void *q = nullptr, *nf = nullptr, *lq = nullptr, *lqs = nullptr, *e12 = nullptr, *lam = nullptr, *g = nullptr,
         *tu = nullptr, *Q = nullptr, *S = nullptr;
    double *partials = nullptr;
    int nblocks = 0;
    double *coef = nullptr;
    int K = 0;
    double *kvec = nullptr, *rho = nullptr, *skn = nullptr;
    // S(k), mixed precision: per-dimension phase tables for the box they were built for
    // STRU_FACTOR Chemical: type-weight parameters, the table built from the
    // types of mtd_set_types, and the per-atom weights (sorted order)
    bool chem = false, wchem = false;
    double chem_ctarget = 0.0, chem_sigma = 1.0;
    std::vector<std::pair<int, double>> chem_map;
    double *d_wtab = nullptr;
    int ntab = 0;
    void *w = nullptr;
};

template <typename P> cudaError_t dalloc(P **p, size_t bytes) {
    *p = nullptr;
    return cudaMalloc((void **)p, bytes < 16 ? 16 : bytes);
}
template <typename P> void dfree(P *&p) {
    if (p) cudaFree((void *)p);
    p = nullptr;
}

constexpr int kHillCap = 4096;

}  // namespace ctx
}  // namespace mtd

using namespace mtd;
using namespace mtd::ctx;

constexpr int kOutSlots = 4;
struct OutSlot {
    double out[64];
    DevStatus status;
    unsigned long long nhills;
    double vir[8];
};
struct PendingOut {
    int slot;
    long long step;
    bool virial;
};

struct mtd_ctx {
    int fp64 = 0;
    int device = 0;
    double boltz = 8.617343e-5;
    GroupTable groups;
    std::string hills_path = "HILLS";
    std::string work_dir;
    Config cfg;
    std::vector<std::string> symnames;
    std::vector<std::vector<ExprInstr>> code;
    cudaStream_t st = nullptr;
    bool box_set = false;
    double lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};
    int periodic[3] = {1, 1, 1};
    bool initialized = false;
    int n = 0, npad = 0, cap_n = 0, n_plan = -1;
    double *d_x = nullptr, *d_fin = nullptr, *d_fout = nullptr;
    int *d_mask = nullptr, *d_image = nullptr;
    int *cellof = nullptr, *slot = nullptr, *perm = nullptr, *smask = nullptr, *arrival = nullptr;
    int *iperm = nullptr;                // caller index -> sorted slot
    double *xs = nullptr;
    float4 *pf = nullptr;
    int *count = nullptr, *start = nullptr;
    int cap_cell = 0;
    std::vector<Env> envs;
    std::vector<Unit> units;
    BiasPlan plan{};
    BiasPlan *d_plan = nullptr;
    bool plan_dirty = true;
    double *d_grid = nullptr;
    long long grid_size = 0;
    HillRec *d_hills = nullptr;
    unsigned long long *d_nhills = nullptr;
    double *d_out = nullptr;
    DevStatus *d_status = nullptr;
    double *d_vpart = nullptr;
    int cap_vpart = 0;
    double *d_vir = nullptr;
    // Pinned outputs of a step.  A context owns kOutSlots of them: the device
    // path writes step t into slot t mod kOutSlots and collects it once its
    // event has completed, so the host never waits for the step it just
    // enqueued; h_out / h_status / h_vir / h_nhills point at the slot in use.
    OutSlot *h_slots = nullptr;
    cudaEvent_t slot_ev[kOutSlots] = {};
    bool ring = true;                    // false for walkers (fixed slot 0, captured in their graph)
    int slot_next = 0;
    std::deque<PendingOut> fifo;         // steps enqueued and not yet collected, oldest first
    unsigned overflow_seen = 0;          // largest neighbour count of an overflowed step drained since mtd_sync
    double *h_out = nullptr;
    DevStatus *h_status = nullptr;
    double *h_vir = nullptr;
    HillRec *h_hills = nullptr;
    unsigned long long *h_nhills = nullptr;
    unsigned long long hills_written = 0;
    std::vector<double> cv;
    double bias = 0.0;
    double virial[6] = {0, 0, 0, 0, 0, 0};
    FILE *f_hills = nullptr;
    FILE *f_rec = nullptr;
    std::string err;
    int launches = 0;
    bool want_virial = false;
    bool pending = false;
    long long pending_step = 0;
    CellGrid last_grid{};
    SysDev last_sys{};
    cudaStream_t own_st = nullptr;
    cudaStream_t side_st = nullptr;      // host -> device force upload beside the CV passes
    bool zc_on = false;                  // this step's force pass writes pinned host f in caller order
    int host_copy_mode = 0;              // mtd_set_host_copy_mode (0: chosen by timing)
    // mode 0: the first eligible mtd_post_force calls try modes 1-3 in turn
    // (wall time of each call), then the mode with the fastest call is kept
    int copy_pick = 0;                   // the mode chosen (0: still trying)
    int copy_calls = 0;                  // eligible calls seen while trying
    int copy_used = 0;                   // mode of the call in progress (0: not eligible)
    double copy_ms[4] = {0, 0, 0, 0};
    int copy_cnt[4] = {0, 0, 0, 0};
    // hill-list bias (CV_dim 4 or NN_BIAS 1): hills, exact sum, learned bias
    mtd_nnbias *nb = nullptr;
    double *d_vdv = nullptr;             // V, dV/ds at this step's s
    WalkState *d_ws1 = nullptr;          // CV values, chain factors and block-sum totals of the last step
    int h_fit = 0;                       // hills the network was fitted on
    bool nn_usable = false;
    cudaEvent_t f_ready = nullptr;
    // atom types (caller order) for STRU_FACTOR Chemical, from mtd_set_types
    int *d_types = nullptr;
    int types_cap = 0, types_n = -1;
    // kernel shapes chosen by mtd_autotune (every choice gives bitwise-identical results)
    int tune_nbr = 0;                    // neighbour search: 0 fast/256, 1 fast/128, 2 flat/128
    int tune_q = 0, tune_l = 0;          // threads per block of the q and lambda passes (0: 256)
    int tune_qsplit = 0;                 // skin lists: the q pass's filter in its own loop (1) or merged (0)
    int tune_skq = 8, tune_skqf = 2;     // S(k): k-vectors per pass of the value pass, unroll of the force pass
    // per-atom dCV/dx export (compute metad/atom): last step's inputs, cached result
    const double *last_x = nullptr;
    const int *last_mask = nullptr;
    long long step_gen = 0;              // steps enqueued so far
    long long dcv_gen = -1;              // step the cached dCV/dx belongs to
    std::string dcv_cal;
    std::vector<double> h_dcv;           // [n][3], caller order
    double *d_dcv = nullptr;             // [2][cap][3]: zero input, gradient output
    int dcv_cap = 0;
    Prof prof;
    bool prof_created = false;
    std::map<std::string, std::pair<long long, double>> prof_total;
    // domain decomposition (mtd_set_domain): caller indices from nown on are ghosts
    int nown = -1;                       // -1: off, every atom is owned
    int dom_rank = 0;
    mtd_allreduce_fn dom_fn = nullptr;
    mtd_allreduce_device_fn dom_dev_fn = nullptr;   // stream-ordered variant (no host round trip)
    void *dom_user = nullptr;
    double *d_xchg = nullptr;            // this rank's unit totals, then the totals over all ranks
    double *h_xchg = nullptr;            // pinned staging of the same
    int xchg_n = 0;
    // two-call step (mtd_set_positions_f64, then mtd_step)
    int staged_n = -1;                   // atoms uploaded and not yet stepped (-1: none)
    bool staged_mask = false;
    int fix_groupbit = 1;
    // skin lists (NEIGH_SKIN > 0): candidate lists and the sorted order kept across steps
    SkinState *d_skin = nullptr;
    GridBar *d_rbar = nullptr;            // grid barrier of the one-launch skin-list rebuild
    int rebuild_limit = 1 << 22;          // its polls per wait (mtd_neighbor_set_wait)
    int rebuild_stall = 0;                // diagnostics: the next rebuild's waits run out
    double *xref = nullptr;              // sorted raw coordinates at the last rebuild
    bool skin_valid = false;             // the kept sorted order and candidates match n and the grid
    int skin_n = -1;
    CellGrid skin_grid{};
    bool skin_last = false;              // the last step used the skin lists
    std::vector<char> env_fused;         // skin lists: environment filtered inside its STEINH L unit's q pass
    bool skin_reset_pending = false;     // the step's first fused q pass closes the skin gate
    unsigned overflow_cand_seen = 0;     // largest candidate count of an overflowed step drained since mtd_sync
};

namespace mtd {
namespace ctx {

mtd_status fail(mtd_ctx *c, mtd_status s, const std::string &m);
mtd_status cuda_check(mtd_ctx *c, cudaError_t e, const char *what);

#define MTD_CU(expr, what)                                        \
    do {                                                          \
        mtd_status _s = cuda_check(c, (expr), what);              \
        if (_s != MTD_OK) return _s;                              \
    } while (0)

// context.cu
size_t real_size(const mtd_ctx *c);
int record_stride(const mtd_ctx *c, const Unit &u);
void use_slot(mtd_ctx *c, int k);
CellGrid make_grid(const mtd_ctx *c, double extra = 0.0);
// Skin lists apply (NEIGH_SKIN > 0, every periodic side >= 2 (cutoff + skin)
// and >= 3 cells of cutoff + skin): the step's cell grid into g either way.
bool skin_grid(const mtd_ctx *c, CellGrid &g);
// Grows the lists a step reported too small: exact lists to hold `need`
// neighbours, skin candidate lists `cand_need` (which forces a rebuild).
mtd_status grow_lists(mtd_ctx *c, unsigned need, unsigned cand_need);
NeighSpec neigh_spec(const Env &e);
SkDev sk_dev(mtd_ctx *c, Unit &u, const double *x, const int *mask);
int estimate_M(const mtd_ctx *c, double rc, int n);
mtd_status alloc_env(mtd_ctx *c, Env &e, int npad);
mtd_status alloc_cand(mtd_ctx *c, Env &e, int npad);
mtd_status alloc_unit(mtd_ctx *c, Unit &u, int npad);
mtd_status ensure_capacity(mtd_ctx *c, int n);
// Host -> device copy from pinned memory in pieces of at most 3 MB: one
// multi-megabyte cudaMemcpyAsync moves ~25 GB/s over the host link, pieces of
// a few MB back to back reach ~50 GB/s.
cudaError_t h2d_pieces(void *dst, const void *src, size_t bytes, cudaStream_t st);
mtd_status ensure_cells(mtd_ctx *c, int ncell);
void build_plan(mtd_ctx *c);
mtd_status plan_units(mtd_ctx *c);
int owned(const mtd_ctx *c);
NeighDev env_dev(const Env &e);
SysDev sys_dev(mtd_ctx *c, const double *x, const int *mask, const int *image);
template <typename T> void run_values(mtd_ctx *c, const CellGrid &g, const double *x, const int *mask);
template <typename T>
void run_forces(mtd_ctx *c, const SysDev &s, const CellGrid &g, const double *x, const int *mask, const double *fin,
                double *fout, bool virial);
void prof_collect(mtd_ctx *c);

// The step's kernels use programmatic dependent launch (kernels.h).
struct PdlScope {
    PdlScope() { pdl_set(true); }
    ~PdlScope() { pdl_set(false); }
};

struct ProfScope {
    Prof *prev;
    explicit ProfScope(mtd_ctx *c) : prev(prof_get()) {
        if (c->prof.on) {
            if (c->prof.n > kProfMax - 64) prof_collect(c);
            prof_set(&c->prof);
            prof_mark("start", c->st);
        }
    }
    ~ProfScope() { prof_set(prev); }
};

mtd_status enqueue_values(mtd_ctx *c, int n, const double *x, const int *mask, const int *image);
mtd_status enqueue_forces(mtd_ctx *c, long long step, const double *x, const int *mask, const double *fin,
                          double *fout, bool virial);
mtd_status enqueue_step(mtd_ctx *c, long long step, int n, const double *x, const int *mask, const int *image,
                        const double *fin, double *fout, bool virial, cudaEvent_t f_ready = nullptr);
mtd_status collect(mtd_ctx *c);
template <typename T>
mtd_status walk_desc(mtd_ctx *c, int n, const double *x, double *f, WalkDesc<T> &d, bool *ok);
mtd_status drain(mtd_ctx *c, bool block);

// decomp.cu
mtd_status exchange_totals(mtd_ctx *c);

// hills.cu
void write_hill_line(mtd_ctx *c, const HillRec &h);
mtd_status list_add_hills(mtd_ctx *c, const std::vector<HillRec> &recs);
std::string path_in(const mtd_ctx *c, const std::string &p);
mtd_status replay_records(mtd_ctx *c, const std::vector<HillRec> &recs);
mtd_status read_hills(mtd_ctx *c, const std::string &path, std::vector<HillRec> &recs, bool *exists);

// autotune.cu
mtd_status autotune_idle(mtd_ctx *c, int n, const double *d_x, const int *d_mask, int reps, int *choice);

}  // namespace ctx
}  // namespace mtd
