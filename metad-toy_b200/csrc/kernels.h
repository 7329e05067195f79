// kernels.h -- device data layouts and the host-side launchers of every kernel.
//
// Layout in HBM (n atoms, npad = n rounded up to the block size):
//   caller order : x_in, f_in, f_out (FP64 AoS n*3), mask, image (int n)
//   sorted order : atoms counting-sorted by cell (z fastest); perm[k] = caller
//                  index of sorted atom k; xs (FP64 AoS raw coordinates for
//                  exact decisions), pf (float4: FP32 offset from the cell's
//                  lower corner + packed cell coordinates), smask
//   neighbours   : ELL index lists, slot-major int[M][npad] (a warp reads 32
//                  consecutive entries per slot); count[npad]; displacements
//                  are recomputed from pf in every pass (4 B per pair instead
//                  of a 16 B record keeps the step's working set near L2 size)
//   per-atom CV  : AoS records of SQ reals (q_lm, LQ_lm, lambda ...) so one
//                  neighbour gather touches one or two 128-byte lines
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"
#include "expr.h"
#include "geo.cuh"

namespace mtd {

struct CellGrid {
    int nc[3];
    int ncell;          // cell keys (with tiles: tiles x 64, the cells of partial tiles stay empty)
    int periodic[3];
    double L[3], invL[3], lo[3], h[3], inv_h[3];
    float hf[3], Lf[3], invLf[3];
    // tiled = 1: cells are keyed (and atoms sorted) by 4 x 4 x 4 tiles of
    // cells (nt tiles per dimension, tile-major, then x, y, z inside a tile),
    // so a block of consecutive atoms is a compact piece of space and its
    // neighbours' records are shared by its own threads; 0: row-major
    // (x, y, z with z fastest), used where a periodic side has fewer than
    // three cells (the general search walks runs of z cells)
    int tiled, nt[3];
};

// Key of cell (x, y, z): the index of its atom range in the sorted order.
__host__ __device__ inline int cell_key(const CellGrid &g, int x, int y, int z) {
    if (!g.tiled) return (x * g.nc[1] + y) * g.nc[2] + z;
    return ((((x >> 2) * g.nt[1] + (y >> 2)) * g.nt[2] + (z >> 2)) << 6) | ((x & 3) << 4) | ((y & 3) << 2) | (z & 3);
}

__host__ __device__ inline GeoF geo_f(const CellGrid &g, const float4 *pf) {
    GeoF r;
    r.pf = pf;
    for (int c = 0; c < 3; ++c) {
        r.hf[c] = g.hf[c];
        r.Lf[c] = g.Lf[c];
        r.invLf[c] = g.invLf[c];
        r.nc[c] = g.nc[c];
        r.periodic[c] = g.periodic[c];
    }
    return r;
}
__host__ __device__ inline GeoD geo_d(const CellGrid &g, const double *xs) {
    GeoD r;
    r.xs = xs;
    for (int c = 0; c < 3; ++c) {
        r.L[c] = g.L[c];
        r.invL[c] = g.invL[c];
        r.periodic[c] = g.periodic[c];
    }
    return r;
}
template <typename T> Geo<T> make_geo(const CellGrid &g, const float4 *pf, const double *xs);
template <> inline Geo<float> make_geo<float>(const CellGrid &g, const float4 *pf, const double *) {
    Geo<float> r;
    r.g = geo_f(g, pf);
    return r;
}
template <> inline Geo<double> make_geo<double>(const CellGrid &g, const float4 *, const double *xs) {
    Geo<double> r;
    r.g = geo_d(g, xs);
    return r;
}

// Skin lists (NEIGH_SKIN): candidate lists built at cutoff + skin are kept
// across steps.  Every step k_refresh repacks the positions in the kept
// sorted order and sets `gate` when a rebuild is due (an atom moved more than
// skin / 2 since the build, a non-finite position, `age` reached NEIGH_EVERY,
// or the host forced it); the rebuild kernels return at once while the gate
// is closed.  The first kernel after them updates age / builds and clears the
// gate for the next step.
struct SkinState {
    unsigned int gate;            // 1: this step rebuilds the cell list and candidate lists
    unsigned int age;             // steps the current candidate lists have served
    unsigned int builds;          // rebuilds so far
    unsigned int invalid;         // a rebuild gave up (grid-barrier wait): the next step rebuilds from scratch
};

struct SysDev {
    int n, npad;
    const double *x;      // caller order, AoS n*3
    const int *mask;      // caller order, may be null (all groups)
    const int *image;     // caller order, may be null
    int *cellof, *slot, *count, *start, *perm, *smask;
    int *iperm;           // caller index -> sorted slot (null: not kept)
    int *arrival;         // [n] atoms by cell in atomic arrival order (cell-list scratch)
    int nown;             // caller indices >= nown are ghosts (domain decomposition): their
                          // sorted group mask is 0, so they are neighbours and never centres
    double *xs;           // sorted raw coordinates AoS npad*3
    float4 *pf;           // sorted cell-relative coordinates + packed cell
    DevStatus *status;    // k_bin flags non-finite positions (bad_pos)
    SkinState *skin;      // skin lists: the rebuild kernels are gated on skin->gate (null: every step)
    double *xref;         // skin lists: sorted raw coordinates at the last rebuild (AoS npad*3)
};

// Neighbour criteria (the reference's per-CV filters).
enum NeighKind {
    NK_RANGE = 0,    // 1e-12 <= r2 <= rc2           (STEINH Q :1358, STRU_FACTOR :1048)
    NK_STEP = 1,     // r2 <= rc2 and r < r0         (STEINH L with a STEP switch)
    NK_SWITCH = 2,   // r2 <= rc2 and sw(r) >= eps   (STEINH L, Local.cu:1257-1262)
    NK_CAND = 3      // skin-list candidates: FP32 r2 <= hi2 (a superset of cutoff + skin)
};

// The FP32 distance decides a candidate when it is outside [lo2, hi2]; inside
// the band (|r^2 - bound| ~ 1e-5 relative) the FP64 test on raw coordinates
// decides, so the neighbour sets equal the FP64 criterion exactly.
struct NeighSpec {
    int kind;
    double rc2;         // exact FP64 list bound
    double r0;          // STEP threshold (r < r0)
    double eps;
    SwParams sw;
    float lo2, hi2;     // FP32 accept-below / reject-above
    int cap;            // STEINH Q cutoff_Natoms, 0 = none
    int variant;        // kernel shape of the fast path (0, 1, 2: see launch_neighbors); same lists
};

struct NeighDev {
    int *list;          // [M][npad] sorted neighbour indices (bit kFlagBit: kept by the centre's cap)
    int *count;         // [npad] neighbours found (may exceed M: overflow)
    double *key_r2;     // STEINH Q: r2 of the last kept neighbour (inf when cap not binding)
    int *key_id;        // STEINH Q: caller index of the last kept neighbour
    int *nkept;         // STEINH Q: min(count, cap)
    int M;
};

// ------------------------------------------------------------------ per-kernel timing
// When a context enables profiling, every launcher records a CUDA event after
// each kernel on the launch stream; consecutive events bracket one kernel.
constexpr int kProfMax = 1024;   // marks of several steps, read back when the buffer is nearly full
struct Prof {
    bool on = false;
    int n = 0;
    cudaEvent_t ev[kProfMax];
    const char *name[kProfMax];
};
void prof_set(Prof *p);                          // active profiler of this host thread (null: off)
Prof *prof_get();
void prof_mark(const char *name, cudaStream_t st);

// ------------------------------------------------------------------ programmatic dependent launch
// Inside a context's step the kernels are launched with the programmatic-
// stream-serialisation attribute: a kernel's blocks may be scheduled while
// the previous kernel's last wave drains, and each kernel waits (pdl_entry)
// for the previous one to complete before reading anything.  Outside a step
// (walkers' graph capture, autotuning) kernels launch plainly and the wait is
// a no-op.
void pdl_set(bool on);                           // this host thread's launches use the attribute
bool pdl_on();
template <typename... KArgs, typename... Args>
void launch_k(void (*kernel)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
              Args &&...args) {
    if (!pdl_on()) {
        kernel<<<grid, block, smem, st>>>(static_cast<KArgs>(args)...);
        return;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// ------------------------------------------------------------------ neighbours
// Cell list (counting sort by cell).  The cell counts must be zero on entry:
// they are zeroed when allocated and again by the scatter pass after use.
// Returns the number of kernels launched.
int launch_build_cells(const CellGrid &g, SysDev &s, cudaStream_t st);
// Neighbour lists from the cell list (ns.kind NK_CAND: skin-list candidates;
// for a cap, the cap selection follows unless ns.kind is NK_CAND).
void launch_neighbors(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev nd, DevStatus *status,
                      cudaStream_t st);
void launch_select_cap(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev nd, cudaStream_t st);
// Skin lists: the per-step repack and rebuild decision (force: the kept
// sorted order is not valid, rebuild without reading it), and the exact
// lists of one environment filtered from its candidates (reset: the first
// kernel after the gated rebuild, which clears the gate).
void launch_refresh(const CellGrid &g, const SysDev &s, int every, double half_skin, int force, cudaStream_t st);
void launch_filter(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev nd, NeighDev cand,
                   DevStatus *status, SkinState *reset, cudaStream_t st);
struct GridBar;
// Skin lists: the gated rebuild (cell list and candidates of one environment,
// fast path) as one cooperative launch with grid barriers (limit: polls per
// wait; stall: diagnostics, one block skips the first barrier).  Co-resident
// blocks of that launch (0: not available, use the separate gated kernels).
int rebuild_blocks();
cudaError_t launch_rebuild(const CellGrid &g, const SysDev &s, const NeighSpec &ns, NeighDev cd, DevStatus *status,
                           GridBar *bar, int limit, int stall, cudaStream_t st);

// ------------------------------------------------------------------ STEINH L
template <typename T> struct LocalDev {
    int n, npad, SQ;
    int LA, LB;                 // orders handled by this unit (LB = 0: single)
    int groupbit;
    SwParams sw_r, sw_cvA, sw_cvB;
    const int *smask;
    const int *perm;
    Geo<T> geo;
    NeighDev nb;
    T *q, *nf, *lq, *lqs, *e12, *lam, *g, *tu;
    double *partials;           // [nblocks][8]: S1A S0A S1B S0B N
    const double *coef;         // c1A c2A c1B c2B (written by the bias kernel)
    int qblock, lblock;         // threads per block of the q and lambda passes (0: kBlock); same results
    // skin lists: the q pass first filters this unit's candidates into nb (filter != 0),
    // in one loop with the sum (qsplit 0) or in a filter loop before it (qsplit 1)
    int filter, qsplit;
    GeoF fgf;                   // FP32 cell-relative positions (the exact decision's first test)
    GeoD fgd;                   // FP64 raw positions (the guard band)
    NeighSpec fspec;
    NeighDev cand;
    DevStatus *status;
    SkinState *reset;           // the first kernel after the gated rebuild: closes the gate
    // force pass over caller indices i0 .. i1 - 1 (iperm: caller -> sorted
    // slot) instead of sorted slots; the same per-atom arithmetic
    const int *iperm;
    int i0, i1;
};
template <typename T> void launch_local_values(const LocalDev<T> &d, cudaStream_t st);
// Reals per STEINH L record (both orders): a multiple of 32 bytes.
int local_record_stride(int LA, int LB, int fp64);
template <typename T>
void launch_local_forces(const LocalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                         double *vpart, DevStatus *status, cudaStream_t st);
// The two force-stage passes separately: lambda, then the force pass (over
// caller indices d.i0 .. d.i1 - 1 when d.iperm is set; no virial then).
template <typename T> void launch_local_lambda(const LocalDev<T> &d, cudaStream_t st);
template <typename T>
void launch_local_force_pass(const LocalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s,
                             const CellGrid &g, double *vpart, DevStatus *status, cudaStream_t st);

// ------------------------------------------------------------------ STEINH Q
template <typename T> struct GlobalDev {
    int n, npad, SQ, L;
    int groupbit, nsw;
    SwParams sw[2];             // SW_FUNC symbols of this CAL
    const int *smask, *perm;
    Geo<T> geo;
    GeoD exact;                 // FP64 raw coordinates for the cap-membership test
    NeighDev nb;
    T *q, *Q;
    double *partials;           // [nblocks][8]: sumQ, sum f1(Q), sum f2(Q), N
    const double *coef;         // c_ave, c_sw1, c_sw2
};
template <typename T> void launch_global_values(const GlobalDev<T> &d, cudaStream_t st);
template <typename T>
void launch_global_forces(const GlobalDev<T> &d, const double *f_src, double *f_dst, const SysDev &s,
                          const CellGrid &g, double *vpart, DevStatus *status, cudaStream_t st);

// ------------------------------------------------------------------ STRU_FACTOR (Debye) and S(k)
template <typename T> struct DebyeDev {
    int n, npad;
    int groupbit;
    double rc2, qf;
    SwParams sw;
    const int *smask, *perm;
    Geo<T> geo;
    NeighDev nb;
    T *S;
    double *partials;           // [nblocks][4]: sumS, sum f(S), N
    const double *coef;         // c_ave, c_count
    T *w;                       // STRU_FACTOR Chemical: per-atom type weight, sorted order (null: all 1)
    const int *types;           // caller-order atom types (Chemical)
    const double *wtab;         // weight of each type 0..ntab-1 (Chemical)
    int ntab;
};
template <typename T> void launch_debye_values(const DebyeDev<T> &d, cudaStream_t st);
template <typename T>
void launch_debye_forces(const DebyeDev<T> &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                         double *vpart, DevStatus *status, cudaStream_t st);

struct SkDev {
    int n, K, groupbit;
    int nown;                   // caller indices >= nown are ghosts (no S(k) term)
    const double *x;            // caller order AoS
    const int *mask;
    const double *k;            // K*3
    double *partials;           // [nblocks][2K]
    int nblocks;
    double *rho;                // 2K (re, im)
    double *ngroup;             // group count
    const double *coef;         // alpha
    int fp64;
    int qv, qf;                 // k-vectors per pass of the value pass (4 / 8 / 16), unroll of the force pass (1 / 2 / 4)
};
void launch_sk_values(const SkDev &d, cudaStream_t st);
void launch_sk_forces(const SkDev &d, const double *f_src, double *f_dst, const SysDev &s, const CellGrid &g,
                      double *vpart, cudaStream_t st);
int sk_blocks(int n);


// ------------------------------------------------------------------ bias grid
enum SymKind {
    SYM_Q_AVE = 0, SYM_Q_SW, SYM_L_MEAN, SYM_L_NSOLID, SYM_L_FRAC, SYM_SF_AVE, SYM_SF_COUNT, SYM_SK_AVE
};

struct SymPlan {
    int kind;
    int unit;        // index in the unit table
    int slot;        // l slot (0/1) for STEINH L, SW slot for STEINH Q
};

struct UnitPlan {
    int kind;              // CalKind of the unit
    const double *partials;
    int nparts, pstride, nvals;
    double *coef;          // coefficient block written for the force kernels
    const double *rho;     // S(k)
    int K;
    const double *sk_n;
};

struct HillRec {
    long long step;
    double s[kMaxDim];
    double w, sigma;
};

constexpr int kMaxUnits = 16;

struct alignas(16) BiasPlan {
    int D;
    int nbin[3];
    double lo[3], hi[3], dcv[3];
    int band[3];
    double sigma, h0, biasf, temp, kb;
    int wt, pace;
    int nsym;
    SymPlan sym[kMaxSymbols];
    int nunit;
    UnitPlan unit[kMaxUnits];
    int ncode[kMaxDim];
    ExprInstr code[kMaxDim][kMaxExprLen];
    double *grid;
    long long grid_size;
    HillRec *hills;
    int hill_cap;
    unsigned long long *nhills;
    double *out;           // [0..D) s, D: V, D+1: deposited flag, kOutSymOffset..: symbol values,
                           // kOutHillOffset..: the hill recorded last (a HillRec)
    const DevStatus *status;   // a neighbour overflow this step: no deposit, zero force coefficients
    struct WalkState *save;    // when set, the step's block-sum totals are kept here (per-atom gradients)
    const double *gsum;        // domain decomposition: every unit's totals summed over the ranks
                               // ([nunit][8]), used in place of this rank's block partials
};
constexpr int kOutSymOffset = 8;   // out[kOutSymOffset + sym]
constexpr int kOutHillOffset = 48;  // out[kOutHillOffset ..+7): the last HillRec, copied out with the step's outputs
static_assert(kOutSymOffset + kMaxSymbols <= kOutHillOffset && kOutHillOffset * 8 + sizeof(HillRec) <= 64 * 8,
              "output layout");

void launch_bias_step(const BiasPlan *d_plan, long long step, cudaStream_t st);
// Domain decomposition: this rank's totals of every unit ([nunit][8], the
// block partials reduced in the order the bias kernel uses), the rho(k) (2K)
// and atom count of each S(k) unit in unit order, and last this step's
// neighbour-overflow count (0: none) and non-finite-position flag (0: none).
void launch_unit_sums(const BiasPlan *d_plan, double *out, cudaStream_t st);
int unit_sums_count(const BiasPlan &P);
void launch_domain_flag(const double *gflag, DevStatus *status, cudaStream_t st);

// Per-walker state handed between the multi-walker bias kernels.
struct WalkState {
    double s[kMaxDim];
    double hill_w;
    int dep, pad;
    double jac[kMaxDim][kMaxSymbols];
    double usum[kMaxUnits][8];
};
void launch_walk_bias(const BiasPlan *const *d_plans, int nwalk, const long long *d_step, WalkState *ws,
                      cudaStream_t st);
// Walkers sharded over ranks: CVs and heights of this rank's walkers packed
// into kWalkRec-double records (out[nwalk][kWalkRec]); then, with every
// rank's records gathered in rank order (recs[nrec][kWalkRec]), the deposit
// of all hills and this rank's force coefficients.
constexpr int kWalkRec = kMaxDim + 4;
void launch_walk_cvs_pack(const BiasPlan *const *d_plans, int nwalk, const long long *d_step, WalkState *ws,
                          double *out, cudaStream_t st);
void launch_walk_finish(const BiasPlan *const *d_plans, int nwalk, const long long *d_step, const WalkState *ws,
                        const double *recs, int nrec, cudaStream_t st);
void launch_hills_replay(const BiasPlan *d_plan, const HillRec *h, int nh, int ncell, cudaStream_t st);

// ------------------------------------------------------------------ persistent multi-walker step
// One walker's arguments for the single-launch step (walk_step.cu); device
// memory, written by the host before the launch and read-only during it.
template <typename T> struct WalkDesc {
    CellGrid g;
    SysDev s;                   // per-step lists (no skin gate)
    NeighSpec ns;
    NeighDev nd;
    LocalDev<T> ld;
    const double *f_src;
    double *f_dst;
    int nb;                     // 256-atom blocks
    int nchunk;                 // 256-cell chunks of the count scan
    const double *d_out;        // the walker's bias outputs (device) ...
    const DevStatus *d_status;
    const unsigned long long *d_nhills;
    double *h_out;              // ... and their pinned host copies, written at the end of the step
    DevStatus *h_status;
    unsigned long long *h_nhills;
};
// The grid barrier's words (device memory, zero when no launch is in flight).
struct GridBar {
    unsigned int count, gen, err, pad;
};
constexpr int kWalkPersistMax = 1024;   // walkers of one persistent step at most
struct WalkStepArgs {
    int nwalk;
    const int *pa, *pc;         // prefix sums of WalkDesc::nb and ::nchunk over the walkers (nwalk + 1)
    const BiasPlan *const *plans;
    const long long *step;      // the step number (pinned host memory)
    WalkState *ws;
    GridBar *bar;
    int limit;                  // barrier polls before a wait gives up
    int stall;                  // diagnostics: block 0 skips the first barrier (the others' waits run out)
};
// Co-resident blocks of the step kernel for STEINH L orders (LA, LB) in
// precision T (0: no such kernel), and its cooperative launch.
template <typename T> int walk_step_blocks(int LA, int LB, bool step_switch);
template <typename T>
cudaError_t launch_walk_step(int LA, int LB, bool step_switch, const WalkDesc<T> *d_desc, const WalkStepArgs &a,
                             int blocks, cudaStream_t st);

// Hill-list bias (no grid; CV_dim up to 4): the CV values and chain factors
// into ws[0]; then, with V and dV/ds at s from the hill sum or the learned
// bias in vdv (V, dV[0..D)), the deposit record, V += the new hill's height
// (a hill adds its full height and no slope at its own centre) and the force
// coefficients.
void launch_list_cvs(const BiasPlan *d_plan, WalkState *ws, cudaStream_t st);
// Force coefficients of every unit for dCV/dx of one symbol (chain factor 1
// on it, 0 on the others), from the block-sum totals kept in ws[0].
void launch_symbol_coef(const BiasPlan *d_plan, int sym, const WalkState *ws, cudaStream_t st);
void launch_list_finish(const BiasPlan *d_plan, long long step, const WalkState *ws, const double *vdv,
                        cudaStream_t st);
void launch_virial_finalize(const double *vpart, int nparts, double *out6, cudaStream_t st);

}  // namespace mtd
