/*
 * metad_b200.h -- C ABI of libmetad_b200.so, the sm_100a implementation of
 * Metad-toy's metadynamics hot path (STEINH Steinhardt CVs, structure factor,
 * Gaussian-hill bias grid) behind the `fix metad` argument grammar.
 *
 * Every entry point takes plain pointers and sizes.  Each one names the
 * reference interface it replaces (paths inside the Metad-toy project).
 *
 * Threading: one host thread per context; calls on one context are not
 * thread-safe, while different contexts may be driven from different host
 * threads at the same time (the library keeps no shared mutable state
 * between contexts).  Each context owns one CUDA stream and all of its
 * device memory.  Caller arrays are borrowed for the duration of a call
 * only.
 */
#ifndef METAD_B200_H
#define METAD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MTD_ABI_VERSION 1

/* Status codes.  The reference stops the run through error->all() / exit(1)
 * (include/utils/zqc_debug.h:59-78); this library returns a code and keeps a
 * message for mtd_last_error(). */
typedef enum {
    MTD_OK = 0,
    MTD_ERR_INVALID_ARG = 1,
    MTD_ERR_PARSE = 2,
    MTD_ERR_CUDA = 3,
    MTD_ERR_OOM = 4,
    MTD_ERR_NEIGH_OVERFLOW = 5,
    MTD_ERR_TIMEOUT = 6,
    MTD_ERR_NAN = 7,
    MTD_ERR_IO = 8,
    MTD_ERR_UNSUPPORTED = 9
} mtd_status;

/* Per-atom arithmetic.  MIXED: FP32 per-atom/per-pair work, FP64 global sums,
 * grid and well-tempered height.  FP64: everything in double. */
typedef enum { MTD_PREC_MIXED = 0, MTD_PREC_FP64 = 1 } mtd_precision;

typedef struct mtd_ctx mtd_ctx;

typedef struct {
    int precision;                    /* mtd_precision */
    int device;                       /* CUDA device ordinal */
    double boltz;                     /* force->boltz (metal units: 8.617343e-5 eV/K) */
    int n_groups;                     /* LAMMPS group table: name -> bitmask, used by CAL ... <group> */
    const char *const *group_names;
    const int *group_bits;
    const char *hills_path;           /* HILLS file; NULL -> "HILLS"; "" -> no file */
    const char *work_dir;             /* directory for rec.log and relative paths; NULL -> CWD */
} mtd_options;

/* Fills defaults: MIXED, device 0, boltz 8.617343e-5, group "all" -> bit 1. */
void mtd_options_default(mtd_options *opt);

/* Parse the `fix ID group metad ...` arguments (the tokens after the style
 * name, i.e. the reference's arg[3..]) and build a context.
 * Replaces FixMetadynamics::FixMetadynamics (src/core/fix_crystallize.cu:32-302),
 * CVFactory::create (src/core/CVFactory.cu:17-29), Steinhardt::create
 * (src/cvs/CVs_Steinhardt.cu:33-161), Stru_factor::create
 * (src/cvs/CVs_Strufactor.cu:34-237) and SwitchFunction::create
 * (include/utils/zqc_switch_function.h:81-161). */
mtd_status mtd_create(int narg, const char *const *arg, const mtd_options *opt, mtd_ctx **out);

/* Replaces FixMetadynamics::~FixMetadynamics (src/core/fix_crystallize.cu:304-337).
 * mtd_create leaves a context in *out even when it fails, so that
 * mtd_last_error() can report why; destroy it either way. */
void mtd_destroy(mtd_ctx *ctx);

/* Host-only check of the same argument grammar, no GPU touched: returns the
 * status mtd_create would return for a parse error and copies the message
 * into err (errlen bytes).  Same reference lines as mtd_create. */
mtd_status mtd_parse_args(int narg, const char *const *arg, const mtd_options *opt, char *err, int errlen);

/* Host-only evaluation of a DIM expression over named symbol values, with the
 * exact partial derivatives d expr / d symbol (grad, nsym values).  The device
 * evaluates the same bytecode every step.  Replaces the exprtk expression and
 * exprtk::derivative of MetaDimensionManager (src/grids/DimSet.cu:54-97). */
mtd_status mtd_eval_expression(const char *expr, int nsym, const char *const *names, const double *values,
                               double *value, double *grad);

/* Box geometry (domain->boxlo/boxhi, x/y/zperiodic); orthogonal boxes.
 * Replaces the box read in Steinhardt_env::get_env (src/cvs/CVs_Steinhardt.cu:443-446). */
mtd_status mtd_set_box(mtd_ctx *ctx, const double lo[3], const double hi[3], const int periodic[3]);

/* First-run initialisation: allocates the bias grid, replays HILLS when
 * METAD_RESTART 1, opens HILLS for writing/appending.
 * Replaces FixMetadynamics::init (src/core/fix_crystallize.cu:343-378),
 * GH_t0_uniformGrid::init_set_mode/init_hills (src/grids/GH_t0_uniformGrid.cu:74-192). */
mtd_status mtd_init(mtd_ctx *ctx);

/* One MD step on host arrays: computes every CAL, the DIM values, deposits a
 * hill when step % PACE == 0, evaluates V(s) and dV/ds, and subtracts the bias
 * force from f (AoS n*3, in place).  mask: LAMMPS atom->mask (NULL = every
 * atom in every group).  image: LAMMPS packed imageint (default 10-bit layout)
 * used to unwrap x for the virial; NULL = x taken as unwrapped.  virial (6,
 * may be NULL) receives sum over atoms of r (x) delta_f as
 * (xx, yy, zz, xy, xz, yz).
 * Replaces FixMetadynamics::post_force (src/core/fix_crystallize.cu:386-472). */
mtd_status mtd_post_force(mtd_ctx *ctx, int64_t step, int n, const double *x, const int *mask,
                          const int *image, double *f, double virial[6]);

/* Same step on device-resident arrays, enqueued on the context stream without
 * a host synchronisation.  f_in and f_out may alias.  Up to four steps may be
 * in flight: each call collects the outputs of steps that have finished (CVs,
 * bias, HILLS rows) without waiting, and waits only when four are pending (or,
 * with the hill-list bias, for the previous step, whose hill joins the list
 * on the host).  mtd_compute_scalar / _vector report the last collected step;
 * mtd_sync() collects every step and reports device error flags. */
mtd_status mtd_post_force_device(mtd_ctx *ctx, int64_t step, int n, const double *d_x, const int *d_mask,
                                 const int *d_image, const double *d_f_in, double *d_f_out);

/* Waits for the context stream and reports device-side errors (neighbour
 * overflow, NaN forces, timeouts) raised by earlier asynchronous calls. */
mtd_status mtd_sync(mtd_ctx *ctx);

/* The same step in two calls, for callers that hand over positions before
 * the force array (the interface shape of a `mtd_step` driver):
 * mtd_set_positions_f64 copies x (AoS n*3), mask (NULL = every atom in every
 * group) and, when a CAL needs them, type (NULL otherwise) to the device
 * before it returns, so the arrays are borrowed for the call only; groupbit
 * is the fix's own group bit, which the reference's post_force does not
 * apply either (src/core/fix_crystallize.cu:386-472): it is checked to be
 * non-zero and recorded.  mtd_step then runs the step on those positions and
 * f_inout (AoS n*3, -= bias force), writes the CV_dim values to cv_out and
 * the bias energy to bias_energy_out (either may be NULL) and the virial
 * (may be NULL; x taken as unwrapped).  Results equal mtd_post_force on the
 * same arrays bit for bit.  mtd_get_peratom is mtd_extract_peratom for the
 * last step's n atoms. */
mtd_status mtd_set_positions_f64(mtd_ctx *ctx, const double *x, const int *type, const int *mask, int n,
                                 int groupbit);
mtd_status mtd_step(mtd_ctx *ctx, int64_t step, double *f_inout, double *cv_out, double *bias_energy_out,
                    double virial_out[6]);
mtd_status mtd_get_peratom(mtd_ctx *ctx, const char *key, double *out);

/* mtd_create with the deck and options in one struct. */
typedef struct {
    int narg;
    const char *const *arg;           /* the tokens after "metad" */
    mtd_options opt;
} mtd_config;
mtd_status mtd_create_from_config(const mtd_config *cfg, mtd_ctx **out);

/* Thermo output.  Replaces FixMetadynamics::compute_scalar / compute_vector
 * (src/core/fix_crystallize.cu:484-494): bias energy V_b(s) and CV k (0-based). */
double mtd_compute_scalar(const mtd_ctx *ctx);
double mtd_compute_vector(const mtd_ctx *ctx, int k);
int mtd_cv_dim(const mtd_ctx *ctx);

/* Per-atom export for `compute metad/atom` / Fix::extract
 * ("colvar_peratom:<CAL>.<prop>", props stein_q, dcvdx_x/y/z, stru_f,
 * chem_pair_r for WEIGHT_CHEM; nnb = neighbours the CV used, for STEINH Q
 * min(neighbours within cutoff_r, cutoff_Natoms); nrc = neighbours within
 * the list criterion before any cap).
 * Copies n values (caller order) into out.  dcvdx_* is the exact gradient of
 * the CV that the first SYMBOL on <CAL> selects, at the last step's positions
 * (STEINH Q and L, STRU_FACTOR, STRU_FACTOR_K); it re-runs that CAL's force
 * kernels once per step and CAL and is cached, so dcvdx_x/y/z of one step
 * cost one pass.  After mtd_post_force_device it reads the caller's position
 * buffer of that step, which must still hold those positions.
 * Replaces FixMetadynamics::extract (src/core/fix_crystallize.cu:592-613),
 * STEIN_QL::get_peratom_ptr (src/cvs/CVs_Steinhardt.cu:1278-1322),
 * Stru_factor::get_peratom_ptr (src/cvs/CVs_Strufactor.cu:974-979). */
mtd_status mtd_extract_peratom(mtd_ctx *ctx, const char *key, double *out, int n);

/* The last step's neighbour lists of CAL `cal` (STEINH Q / L, STRU_FACTOR),
 * caller order: counts[i] (n values) = neighbours atom i's CV terms use (for
 * STEINH Q the cutoff_Natoms nearest within cutoff_r, ties by caller index;
 * for STEINH L those with sigma(r) >= cutoff_eps; for STRU_FACTOR those within
 * cutoff_r).  idx may be NULL; otherwise idx[i * max_per_atom + t] receives
 * their caller indices in ascending order, -1 padded, and a count above
 * max_per_atom returns MTD_ERR_INVALID_ARG.  Replaces the reference's
 * per-atom list and counts d_calculated_numneigh, d_neigh_both_in_r_N and
 * d_neigh_in_cutoff_r of get_environment_Steinhardt_Q
 * (src/cvs/CVs_Steinhardt.cu:1324-1406) and the lists of
 * get_environment_Steinhardt_LocalQ (src/cvs/CVs_Steinhardt_Local.cu:1210-1285). */
mtd_status mtd_get_neighbors(mtd_ctx *ctx, const char *cal, int n, int *counts, int *idx, int max_per_atom);

/* Skin lists (the `fix metad` extension keywords NEIGH_SKIN s and NEIGH_EVERY
 * k): neighbour candidates within cutoff + s are kept across steps and
 * filtered to the exact lists every step; the cell list and the candidates
 * are rebuilt when an atom has moved more than s / 2 since the last rebuild,
 * when a position is not finite, when the atom count or the box changes, and
 * at least every k steps (k = 0: only then).  The neighbour sets equal the
 * per-step ones exactly (the sums may differ in their last bits: the
 * neighbours come in another order).  rebuilds receives the rebuilds so far,
 * skin_active whether the last step used skin lists (they apply where every
 * periodic side is at least 2 (cutoff + s) and holds 3 cells of cutoff + s).
 * The reference reads LAMMPS's skin lists and filters them by r < cutoff_r
 * every step (src/cvs/CVs_Steinhardt.cu:135-147, src/core/neigh_hub.cu:191-222). */
mtd_status mtd_neighbor_stats(mtd_ctx *ctx, int64_t *rebuilds, int *skin_active);

/* Skin lists: the rebuild (cell list and candidate lists) runs as one
 * cooperative launch whose phases are separated by grid barriers.  Every
 * barrier wait polls at most `limit` times (0: the default, 4,194,304) before
 * it gives up; a rebuild that gave up makes that step return MTD_ERR_TIMEOUT
 * (no hill deposited, no bias force applied) and the next step rebuild from
 * scratch.  stall = 1 (diagnostics) makes the next rebuild's waits run out.
 * Extension (the reference has no device-side rebuild). */
mtd_status mtd_neighbor_set_wait(mtd_ctx *ctx, int limit, int stall);

/* How mtd_post_force / mtd_step move f (n x 3 FP64) over the host link when
 * f is pinned host memory, the deck has one STEINH L unit and no virial is
 * asked for (otherwise mode 1 applies):
 *   1  f uploaded on a side stream during the CV passes, downloaded after;
 *   2  f uploaded as in 1, written back by the force pass itself (zero copy,
 *      one thread per caller index so every warp writes one contiguous
 *      stretch), no download;
 *   3  f read and written in place by the force pass (zero copy both ways).
 * 0 (default): the fastest depends on the host platform (measured: mode 3 on
 * some hosts, mode 1 on others), so the first eligible calls of
 * mtd_post_force run modes 1-3 in turn (three timed calls each, after one
 * warm-up call) and the mode with the fastest call is kept; setting
 * 0 again starts a new trial.  Forces are bitwise identical in every mode.
 * Extension (no counterpart). */
mtd_status mtd_set_host_copy_mode(mtd_ctx *ctx, int mode);

/* The host copy mode in use: the caller's, or the one the trial of mode 0
 * picked (0 while the trial runs).  Extension (no counterpart). */
mtd_status mtd_host_copy_mode_in_use(mtd_ctx *ctx, int *mode);

/* Replays a HILLS file into the grid (rows `step cv[D] height sigma`).
 * Replaces GH_t0_uniformGrid::init_hills (src/grids/GH_t0_uniformGrid.cu:101-192). */
mtd_status mtd_hills_replay(mtd_ctx *ctx, const char *path);

/* Copies the bias grid (FP64, row-major, dimension 0 slowest) to host. */
mtd_status mtd_get_grid(mtd_ctx *ctx, double *out, int64_t count);

/* Number of device kernels the last step launched (diagnostics). */
int mtd_last_launch_count(const mtd_ctx *ctx);

/* Runs the context's work on an external CUDA stream (a cudaStream_t, e.g. the
 * host code's or LAMMPS/Kokkos's stream); NULL returns to the context's own
 * stream.  The reference runs everything on the default stream
 * (src/cvs/CVs_Steinhardt.cu:1110). */
mtd_status mtd_set_stream(mtd_ctx *ctx, void *cuda_stream);

/* Per-kernel timing with CUDA events recorded after every launch.  enable
 * resets the totals; each step then synchronises on its last event and adds
 * every kernel's duration to a per-name total.  mtd_profile_report writes
 * lines "name calls total_ms\n" into buf and returns the bytes needed.
 * The reference has no timers (its only timing is LAMMPS's Modify time). */
mtd_status mtd_profile_enable(mtd_ctx *ctx, int enable);
int mtd_profile_report(mtd_ctx *ctx, char *buf, int len);

/* Autotuner: times the interchangeable kernel shapes on device positions
 * d_x (n x 3, caller order; d_mask may be NULL) over `reps` launches each and
 * keeps the fastest -- the neighbour search (0: 256-thread blocks, 1:
 * 128-thread blocks, 2: flat per-thread candidate loop) and the threads per
 * block of the q and lambda passes (256 or 128).  Every shape gives
 * bitwise-identical results, so tuning never changes a step's output; it
 * records no step and deposits nothing.  choice (may be NULL) receives the
 * three picks.  mtd_set_tuning sets them directly (q/lambda 0 = 256).
 * No counterpart in the reference (fixed launch shapes). */
mtd_status mtd_autotune(mtd_ctx *ctx, int n, const double *d_x, const int *d_mask, int reps, int choice[3]);
mtd_status mtd_set_tuning(mtd_ctx *ctx, int neighbor_shape, int q_block, int lambda_block);

/* Shapes of the STRU_FACTOR_K passes, chosen by mtd_autotune when the deck
 * has that CAL: k-vectors per pass over the atoms of the value pass (4, 8 or
 * 16: a register tile of partial sums) and the unroll depth of the force
 * pass's loop over k (1, 2 or 4).  Every k is summed in the same order
 * whatever the shape, so the results are bitwise identical.  Defaults 8, 2. */
mtd_status mtd_sk_tiles(mtd_ctx *ctx, int *q_values, int *q_force);
/* Every tuned shape: neighbour search, q block, lambda block (0 = 256),
 * skin-list q pass with its filter in a separate loop (1) or merged with the
 * sum (0), S(k) value-pass k-tile and force-pass unroll. */
mtd_status mtd_get_tuning(mtd_ctx *ctx, int out[6]);
mtd_status mtd_set_tuning_all(mtd_ctx *ctx, const int in[6]);
mtd_status mtd_set_sk_tiles(mtd_ctx *ctx, int q_values, int q_force);

/* Atom types (caller order, n values, host array) for `STRU_FACTOR ...
 * Chemical` and `WEIGHT_CHEM`, whose pair terms are weighted by
 * w(type_i) w(type_j): w from the
 * CAL's Chem_map pairs, else exp(-(type - Chem_ctarget)^2 / (2 Chem_sigma^2)),
 * type 0 weighing 0.  Call it before the first step and whenever types or
 * atom order change; a step with a Chemical CAL and no types for its n atoms
 * fails.  mtd_needs_types tells whether the context has such a CAL.
 * Replaces the type upload of Stru_fact_chem_env::refresh_lmpbox and its
 * weight table (src/cvs/CVs_Strufactor_chem.cu:33-55, :77-100). */
mtd_status mtd_set_types(mtd_ctx *ctx, int n, const int *types);
int mtd_needs_types(const mtd_ctx *ctx);

/* Domain decomposition across ranks (one context per rank).  After
 * mtd_set_domain, the n atoms of every step are this rank's nlocal owned
 * atoms followed by ghosts (images of other ranks' atoms and periodic images,
 * supplied by the caller): ghosts are neighbours only, never centres of a CV
 * sum.  The box is the caller's subdomain grown by mtd_ghost_cutoff() on each
 * side, normally with periodic = {0,0,0} (the ghosts carry the images).
 * Once per step, between the CV passes and the bias, the library calls
 * fn(buf, count, user) with this rank's totals (unit sums, S(k) sums, a
 * neighbour-overflow flag and a non-finite-position flag; count is the same
 * on every rank); fn must replace buf with
 * the element-wise sum over all ranks, the same bits on every rank
 * (MPI_Allreduce(MPI_IN_PLACE, buf, count, MPI_DOUBLE, MPI_SUM, world)), and
 * return 0.  Every rank then holds the same CVs, deposits the same hill and
 * keeps the same grid; rank 0 alone writes HILLS and the record file.  The
 * forces written to f cover all n rows: a ghost row holds the bias force of
 * this rank's centres on that image, which the caller adds to the owning
 * atom (LAMMPS reverse communication).  The virial is this rank's share.  A
 * neighbour overflow on any rank makes every rank retry the step together; a
 * NaN or Inf position on any rank makes every rank skip the deposit and the
 * bias force and return MTD_ERR_NAN, so the ranks stay in step.
 * Call before the first step; mtd_set_nlocal updates nlocal when atoms
 * migrate.  Needs the grid bias (not the hill-list bias).
 * Replaces the per-rank reductions of the reference's CVs under LAMMPS's
 * decomposition: MPI_Allreduce of the local sums over nlocal atoms
 * (src/cvs/CVs_Steinhardt.cu:836, src/cvs/CVs_Strufactor.cu:653, :671,
 * src/cvs/CV_Weighted_Chemical_Pair_Order.cu:306, :324) with ghosts
 * nlocal..nlocal+nghost (src/cvs/CVs_Steinhardt.cu:595).  The reference's
 * forward communication of per-atom CV values to ghosts before the gradient
 * (src/cvs/CVs_Strufactor.cu:805-808) is not needed: each rank applies only
 * its own centres' terms, to owned and ghost rows alike, and the ghost rows
 * go back through the fix's reverse communication
 * (src/core/fix_crystallize.cu:510-520). */
typedef int (*mtd_allreduce_fn)(double *buf, int count, void *user);
mtd_status mtd_set_domain(mtd_ctx *ctx, int nlocal, int rank, mtd_allreduce_fn fn, void *user);
/* The same with the exchange kept on the device: fn(d_buf, count, stream,
 * user) receives the totals in device memory and must enqueue, on `stream`
 * (the context's cudaStream_t), their in-place sum over the ranks, e.g.
 * ncclAllReduce(d_buf, d_buf, count, ncclFloat64, ncclSum, comm, stream),
 * and return 0.  The step then continues on the stream with no host
 * synchronisation (the host callback costs one device-to-host and one
 * host-to-device copy and a stream synchronisation per step). */
typedef int (*mtd_allreduce_device_fn)(double *d_buf, int count, void *stream, void *user);
mtd_status mtd_set_domain_device(mtd_ctx *ctx, int nlocal, int rank, mtd_allreduce_device_fn fn, void *user);
mtd_status mtd_set_nlocal(mtd_ctx *ctx, int nlocal);
/* Ghost shell the caller must supply under domain decomposition: cutoff_r of
 * STEINH Q and STRU_FACTOR, 2 x the cutoff of STEINH L (its centres read q_lm
 * of neighbours, which need their own neighbours), 0 for S(k) alone; with
 * skin lists (NEIGH_SKIN s) the shell grows by s, and the ghost atoms chosen
 * with it should stay the same between rebuilds (as LAMMPS keeps its ghosts
 * between reneighborings): a change of the atom count forces a rebuild. */
double mtd_ghost_cutoff(const mtd_ctx *ctx);

/* Largest neighbour count seen by the last step for CAL `name` (cap reporting). */
int mtd_max_neighbors(mtd_ctx *ctx, const char *name);

const char *mtd_last_error(const mtd_ctx *ctx);

/* Hill-list bias state of a context (CV_dim 4 or NN_BIAS 1): hills deposited,
 * hills the learned bias was last fitted on, and whether that fit passed its
 * validation (then V = network + exact sum over the hills since the fit; else
 * the exact sum).  No counterpart in the reference. */
mtd_status mtd_nn_state(const mtd_ctx *ctx, int *hills, int *hills_fitted, int *usable);
int mtd_abi_version(void);

/* k-vector structure factor of a group, computed with NO device allocation.
 * This entry point has no counterpart in the reference.  It is an
 * allocation-free variant of the STRU_FACTOR_K unit of a context:
 *   rho(k) = sum_{i in group} exp(i k.x_i),   S = sum_k |rho(k)|^2 / (N K).
 * For callers that cannot allocate device memory at the point of the call:
 * an MD engine that computes this CV between its own kernels on several
 * streams (cudaMalloc / cudaFree synchronise the device and would serialise
 * them) or that runs with all device memory reserved up front by its own pool.
 *   n, d_x      0 <= n <= INT_MAX atoms, device FP64 AoS n*3 (caller order)
 *   d_mask      device group bitmask per atom, NULL = every atom; groupbit as in mtd_options
 *   nk, d_k     1 <= nk <= 1024 k-vectors, device FP64 AoS nk*3
 *   precision   MTD_PREC_FP64, or MTD_PREC_MIXED: FP32 sincos of the reduced FP64 phase
 *   d_rho       device 2*nk doubles (Re, Im per k) or NULL
 *   d_s         device 1 double: S
 *   stream      cudaStream_t or NULL; the call only enqueues work
 *   err/errlen  optional message buffer
 * Block partials go to a fixed 1 MiB file-scope device array; no part of it
 * has to start at zero (each call writes every entry it reads).  The first
 * call on a device (that device current) resolves the array's address with
 * cudaGetSymbolAddress: make it before any stream capture.  Calls in flight at
 * the same time on one device share the array and race: order them on one
 * stream.  nk outside [1, 1024] returns MTD_ERR_INVALID_ARG. */
mtd_status mtd_sk_noalloc(int n, const double *d_x, const int *d_mask, int groupbit, int nk, const double *d_k,
                          int precision, double *d_rho, double *d_s, void *stream, char *err, int errlen);

/* ---------------------------------------------------------------- multiple walkers
 * nwalk replicas (uneven atom counts, own boxes) that share one bias grid.
 * Every walker is a context built from the same `fix metad` arguments; one
 * step computes all walkers' CVs concurrently, deposits their hills in walker
 * order with WT heights taken from the grid as it stood at the start of the
 * step, then evaluates every walker's V, dV/ds and forces on the updated grid.
 * One HILLS file for the group (rows in walker order per deposit step).
 * No counterpart in the reference (one walker per `fix metad`); the deposit
 * rule is GH_t0_uniformGrid::add_hill (src/grids/GH_t0_uniformGrid.cu:195-208)
 * applied to each walker's hill in turn.  METAD_RESTART is not replayed for a
 * group. */
typedef struct mtd_walkers mtd_walkers;

mtd_status mtd_walkers_create(int nwalk, int narg, const char *const *arg, const mtd_options *opt,
                              mtd_walkers **out);
void mtd_walkers_destroy(mtd_walkers *W);
const char *mtd_walkers_last_error(const mtd_walkers *W);
int mtd_walkers_count(const mtd_walkers *W);
mtd_status mtd_walkers_set_box(mtd_walkers *W, int k, const double lo[3], const double hi[3], const int periodic[3]);
mtd_status mtd_walkers_init(mtd_walkers *W);

/* Walkers sharded over ranks (one walkers object per rank and GPU, each with
 * the same number of walkers nwalk; global walker id = rank * nwalk + k).
 * Every step, after the CVs, each rank's hills (kWalkRec = 8 doubles per
 * walker: s[4], height, deposit flag, overflow flag, 0) are gathered from
 * all ranks in rank order by the caller's allgather -- fn(send, count,
 * recv, user) on host buffers (recv holds nranks * count doubles), or the
 * device variant that enqueues it on the walkers' stream (e.g.
 * ncclAllGather(d_send, d_recv, count, ncclFloat64, comm, stream)) -- and
 * every rank deposits all hills in global walker order, so every rank keeps
 * the same grid.  A neighbour overflow of any walker on any rank makes every
 * rank report the step for repetition.  Rank 0 alone writes HILLS.  Call
 * before the first step; the CUDA graph is not used while sharded.
 * Replaces nothing in the reference (no multi-walker mode); the shape is the
 * hill allgather per PACE step of a walker-sharded run. */
typedef int (*mtd_allgather_fn)(const double *send, int count, double *recv, void *user);
typedef int (*mtd_allgather_device_fn)(const double *d_send, int count, double *d_recv, void *stream, void *user);
mtd_status mtd_walkers_set_ranks(mtd_walkers *W, int rank, int nranks, mtd_allgather_fn fn, void *user);
mtd_status mtd_walkers_set_ranks_device(mtd_walkers *W, int rank, int nranks, mtd_allgather_device_fn fn,
                                        void *user);

/* Capture the step in a CUDA graph (one graph launch per MD step once the
 * atom counts and array pointers repeat); 0 = plain launches. */
mtd_status mtd_walkers_enable_graph(mtd_walkers *W, int enable);

/* One MD step on device arrays: d_x[k] (n[k] x 3 FP64, caller order) and
 * d_f[k] updated in place (f -= dV/dx).  Asynchronous; mtd_walkers_sync
 * collects outputs and device errors (a neighbour overflow grows the lists and
 * asks for the step to be repeated). */
mtd_status mtd_walkers_step_device(mtd_walkers *W, int64_t step, const int *n, const double *const *d_x,
                                   double *const *d_f);
mtd_status mtd_walkers_sync(mtd_walkers *W);
/* Runs mtd_autotune on every walker with its own positions (walker k's three
 * picks into choices[3k..3k+2], may be NULL); the next step re-captures the
 * CUDA graph with the chosen shapes. */
mtd_status mtd_walkers_autotune(mtd_walkers *W, const int *n, const double *const *d_x, int reps, int *choices);
/* One launch per MD step: when every walker holds one STEINH L unit (one or
 * two orders) on one neighbour environment, without skin lists and not
 * sharded over ranks, a step runs as ONE persistent cooperative kernel over
 * all walkers (cell lists, neighbour lists, CVs, the deposit in walker
 * order, V, dV/ds and forces, phases separated by a grid barrier whose every
 * wait is bounded), with the same arithmetic as the per-walker kernels and
 * the same results bit for bit; with the CUDA graph enabled that launch is
 * replayed.  enable 0 selects the per-walker kernels (the path for every
 * other deck).  mtd_walkers_persistent_active tells whether the last step
 * ran as one launch.  No counterpart in the reference. */
mtd_status mtd_walkers_enable_persistent(mtd_walkers *W, int enable);
int mtd_walkers_persistent_active(const mtd_walkers *W);
/* Diagnostics of the persistent step's grid barrier: every wait polls at
 * most `limit` times (0: the default, 2^22) before the step gives up, and
 * mtd_walkers_sync then returns MTD_ERR_TIMEOUT (the step is incomplete and
 * should be repeated); stall = 1 makes one block skip the first barrier so
 * that the others' waits run out (a check of that path), 0 restores normal
 * operation. */
mtd_status mtd_walkers_set_wait(mtd_walkers *W, int limit, int stall);
double mtd_walkers_cv(const mtd_walkers *W, int k, int d);
double mtd_walkers_bias(const mtd_walkers *W, int k);
mtd_status mtd_walkers_get_grid(mtd_walkers *W, double *out, int64_t count);
int mtd_walkers_last_launch_count(const mtd_walkers *W);

/* ---------------------------------------------------------------- learned bias
 * V_theta(s) for CV_dim >= 3, where the grid blows up: an MLP D -> 128 -> 128
 * -> 1 (SiLU, BF16 weights, FP32 accumulation, the 128 x 128 layer and its
 * backward contractions on the tensor cores), trained on the device on the
 * FP64 hill sum of the hills deposited so far.  The exact sum stays the check
 * of its error (mtd_nnbias_validate) and the fallback (use_nn = -1 below).
 * No counterpart in the reference, whose only bias representations are the
 * grids (src/grids/GH_t0_uniformGrid.cu, src/grids/GH_t1_sparseGrid.cu).
 * Hills are isotropic Gaussians h exp(-|s - c|^2 / (2 sigma^2)).  Inputs are
 * normalised over the box [lo, hi]; calls on one object are not thread-safe. */
typedef struct mtd_nnbias mtd_nnbias;

/* 1 <= D <= 4; He-initialised weights from seed.  *out is set even on failure. */
mtd_status mtd_nnbias_create(int D, const double *lo, const double *hi, unsigned long long seed, mtd_nnbias **out);
void mtd_nnbias_destroy(mtd_nnbias *nb);
const char *mtd_nnbias_last_error(const mtd_nnbias *nb);

/* Appends n hills: centres (n*D), heights (n), widths (n). */
mtd_status mtd_nnbias_add_hills(mtd_nnbias *nb, int n, const double *centers, const double *heights,
                                const double *sigmas);
int mtd_nnbias_num_hills(const mtd_nnbias *nb);

/* Exact FP64 hill sum V (npts) and dV/ds (npts*D, may be NULL) at host points (npts*D). */
mtd_status mtd_nnbias_exact(mtd_nnbias *nb, int npts, const double *pts, double *V, double *dV);

/* The network's V and dV/ds at host points, batched on the tensor cores. */
mtd_status mtd_nnbias_eval(mtd_nnbias *nb, int npts, const double *pts, double *V, double *dV);

/* Fit: ntrain sampled points (half near hill centres, half uniform in the box)
 * with exact targets, iters Adam steps (lr, cosine decay over the second half)
 * on minibatches of `batch`; final_loss = mean squared error in V units^2. */
mtd_status mtd_nnbias_fit(mtd_nnbias *nb, int ntrain, int iters, int batch, double lr, unsigned long long seed,
                          double *final_loss);

/* max and RMS of |V_theta - V_exact| on npts sampled points; the network
 * becomes usable (mtd_nnbias_usable) when max <= tol. */
mtd_status mtd_nnbias_validate(mtd_nnbias *nb, int npts, unsigned long long seed, double tol, double *max_err,
                               double *rms_err);
int mtd_nnbias_usable(const mtd_nnbias *nb);

/* Bias at one device-resident point (D doubles) into d_V (1) and d_dV (D),
 * enqueued on `stream` (cudaStream_t, NULL = the object's stream):
 * use_nn = 1 network, 0 exact sum, -1 network if the last validation passed
 * else the exact sum.  One call in flight per object. */
mtd_status mtd_nnbias_point_device(mtd_nnbias *nb, const double *d_s, double *d_V, double *d_dV, int use_nn,
                                   void *stream);

/* Bias at npts device-resident points (rows of D doubles) into d_V (npts) and
 * d_dV (npts rows of D; NULL = values only), enqueued on `stream`; use_nn as
 * above.  The network path keeps grow-only scratch in the object (allocated
 * on the first call of a larger batch).  No counterpart in the reference. */
mtd_status mtd_nnbias_eval_device(mtd_nnbias *nb, int npts, const double *d_pts, double *d_V, double *d_dV,
                                  int use_nn, void *stream);

/* Checks: the FP32 master parameters (17,281 floats: W1[128][4], b1[128],
 * W2[128][128], b2[128], w3[128], b3), the output scale, and one gradient of
 * the mean squared error sum_i (V_theta(s_i)/vscale - t_i/vscale)^2 / npts on
 * given points and targets, without an update. */
/* Waits for the object's stream and reports MTD_ERR_TIMEOUT when a network
 * tile enqueued since the last check (mtd_nnbias_eval_device) gave up a
 * tensor-core wait; work enqueued on another stream must have completed
 * first (synchronise that stream).  Clears the flag. */
mtd_status mtd_nnbias_sync(mtd_nnbias *nb);

/* Diagnostics of the tensor-core waits of the network's tile kernel: every
 * mbarrier wait polls at most `tries` times (0: the default, 2^20) before the
 * tile gives up -- it issues no further MMA, waits once more with the same
 * limit for the batch in flight, releases its tensor memory and the call
 * returns MTD_ERR_TIMEOUT.  stall = 1 makes every tile, after its first
 * tensor-core batch has completed, wait on a barrier phase that nothing
 * completes, so the next batched call takes that path (a check of it that
 * leaves no work in flight); stall = 0 restores normal operation.  No
 * counterpart in the reference. */
mtd_status mtd_nnbias_set_wait(mtd_nnbias *nb, int tries, int stall);

mtd_status mtd_nnbias_get_params(mtd_nnbias *nb, float *out);
mtd_status mtd_nnbias_set_params(mtd_nnbias *nb, const float *in, double vscale);
double mtd_nnbias_vscale(const mtd_nnbias *nb);
mtd_status mtd_nnbias_loss_grad(mtd_nnbias *nb, int npts, const double *pts, const double *targets, double vscale,
                                float *grad, double *loss);

#ifdef __cplusplus
}
#endif
#endif
