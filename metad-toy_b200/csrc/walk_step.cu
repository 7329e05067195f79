// walk_step.cu -- the multi-walker MD step as ONE persistent kernel launch.
//
// Every phase of the step runs for all walkers inside one cooperative launch
// of co-resident blocks, separated by a grid barrier:
//   bin -> cell-count scan (per 256-cell chunk, then the chunk offsets) ->
//   scatter -> place -> neighbour lists -> q_lm -> LQ_lm (block partials) ->
//   walker CVs and WT heights -> the group's deposit in walker order ->
//   V, dV/ds and force coefficients -> lambda -> forces.
// Each phase is a loop over "virtual blocks" of all walkers (256 atoms, 256
// cells or one walker each) and runs the same per-thread bodies as the
// per-walker kernels (neigh_body.cuh, local_body.cuh, the walker bias phases
// of bias.cu), with the same partial-sum blocks, so the results equal the
// per-walker kernels' bit for bit.  The step number and the outputs go
// through pinned host memory, so the step is this one launch.
//
// Grid barrier (persist.cuh): every wait polls at most `limit` times, after
// which the block records the failure and leaves the kernel, and every other
// block leaves at its next barrier (the host reports MTD_ERR_TIMEOUT and
// resets the barrier).  The cooperative launch makes all blocks co-resident,
// so the waits end in normal operation.
//
// The deposit rule is GH_t0_uniformGrid::add_hill
// (src/grids/GH_t0_uniformGrid.cu:195-208) applied to each walker's hill in
// turn, with heights from the grid as it stood at the start of the step.
#include "local_body.cuh"
#include "persist.cuh"

namespace mtd {

// bias.cu
__device__ void walk_phase_cvs(const BiasPlan *const *plans, int w, const long long *d_step, WalkState *ws);
__device__ void walk_phase_deposit(const BiasPlan *const *plans, int nwalk, const long long *d_step,
                                   const WalkState *ws, int vblock, int nvblocks);
__device__ void walk_phase_coef(const BiasPlan *const *plans, int nwalk, int w, const WalkState *ws);

namespace {

constexpr int kWalkBlock = kPersistBlock;

// Virtual block v of a phase -> (walker, block within the walker) from the
// prefix sums pre[0..nwalk].
__device__ __forceinline__ int walker_of(const int *pre, int nwalk, int v) {
    int lo = 0, hi = nwalk;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (pre[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

template <int LA, int LB, typename T, bool STEP>
__global__ void __launch_bounds__(kWalkBlock, 3) k_walk_step(const WalkDesc<T> *__restrict__ wd, WalkStepArgs a) {
    constexpr int KIND = STEP ? NK_STEP : NK_SWITCH;
    __shared__ int pa[kWalkPersistMax + 1], pc[kWalkPersistMax + 1];
    // the step number lives in pinned host memory: one read per block over
    // the host link, every later read from shared memory
    __shared__ long long s_step;
    for (int t = threadIdx.x; t <= a.nwalk; t += blockDim.x) {
        pa[t] = a.pa[t];
        pc[t] = a.pc[t];
    }
    if (threadIdx.x == 0) s_step = *(volatile const long long *)a.step;
    __syncthreads();
    const int nw = a.nwalk;
    const int G = gridDim.x;
    const int tb = pa[nw], tc = pc[nw];
    // cell list
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const CellGrid &g = wd[w].g;
        const SysDev &s = wd[w].s;
        bin_body(g, s, v - pa[w]);
    }
    if (!grid_barrier(a.bar, a.limit, a.stall && blockIdx.x == 0)) return;
    for (int v = blockIdx.x; v < tc; v += G) {
        const int w = walker_of(pc, nw, v);
        const SysDev &s = wd[w].s;
        const int ncell = wd[w].g.ncell;
        scan_chunk(s, ncell, v - pc[w], s.start + ncell + 1);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int v = blockIdx.x; v < tc; v += G) {
        const int w = walker_of(pc, nw, v);
        const SysDev &s = wd[w].s;
        const int ncell = wd[w].g.ncell;
        scan_offset(s, ncell, v - pc[w], wd[w].nchunk, s.start + ncell + 1);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const SysDev &s = wd[w].s;
        scatter_body(s, wd[w].g.ncell, v - pa[w], wd[w].nb);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const CellGrid &g = wd[w].g;
        const SysDev &s = wd[w].s;
        place_body(g, s, v - pa[w]);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    // neighbour lists and CV values
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const CellGrid &g = wd[w].g;
        const SysDev &s = wd[w].s;
        const NeighSpec &ns = wd[w].ns;
        const NeighDev &nd = wd[w].nd;
        neighbors_fast_body<KIND>(g, s, ns, nd, s.status, v - pa[w]);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const LocalDev<T> &d = wd[w].ld;
        local_q_body<LA, LB, T, STEP, false>(d, v - pa[w]);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const LocalDev<T> &d = wd[w].ld;
        local_lq_body<LA, LB, T, STEP>(d, v - pa[w]);
        __syncthreads();
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    // bias: every walker's CVs, the deposit in walker order, coefficients
    for (int w = blockIdx.x; w < nw; w += G) walk_phase_cvs(a.plans, w, &s_step, a.ws);
    if (!grid_barrier(a.bar, a.limit, false)) return;
    // one block deposits: spreading the bins over every block measured slower here
    if (blockIdx.x == 0) walk_phase_deposit(a.plans, nw, &s_step, a.ws, 0, 1);
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int w = blockIdx.x; w < nw; w += G) walk_phase_coef(a.plans, nw, w, a.ws);
    if (!grid_barrier(a.bar, a.limit, false)) return;
    // outputs of every walker to pinned host memory (read after the stream synchronises)
    for (int w = blockIdx.x; w < nw; w += G) {
        const WalkDesc<T> &D = wd[w];
        for (int t = threadIdx.x; t < 64; t += blockDim.x) D.h_out[t] = __ldcg(D.d_out + t);
        if (threadIdx.x < (int)(sizeof(DevStatus) / sizeof(unsigned)))
            reinterpret_cast<unsigned *>(D.h_status)[threadIdx.x] =
                reinterpret_cast<const volatile unsigned *>(D.d_status)[threadIdx.x];
        if (threadIdx.x == 0) *D.h_nhills = *(volatile const unsigned long long *)D.d_nhills;
    }
    // forces
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const LocalDev<T> &d = wd[w].ld;
        local_lambda_body<LA, LB, T, STEP>(d, v - pa[w]);
    }
    if (!grid_barrier(a.bar, a.limit, false)) return;
    for (int v = blockIdx.x; v < tb; v += G) {
        const int w = walker_of(pa, nw, v);
        const LocalDev<T> &d = wd[w].ld;
        const SysDev &s = wd[w].s;
        const CellGrid &g = wd[w].g;
        local_force_body<LA, LB, T, STEP>(d, wd[w].f_src, wd[w].f_dst, s, g, nullptr, s.status, v - pa[w]);
    }
}

template <int LA, int LB, typename T, bool STEP> struct StepKernel {
    static void *fn() { return reinterpret_cast<void *>(&k_walk_step<LA, LB, T, STEP>); }
};

template <typename T> void *step_kernel(int LA, int LB, bool step_switch) {
    const int key = LA * 16 + LB;
#define MTD_WSK(A, B)                                                                                           \
    case A * 16 + B:                                                                                            \
        return step_switch ? StepKernel<A, B, T, true>::fn() : StepKernel<A, B, T, false>::fn();
    switch (key) {
        MTD_WSK(3, 0) MTD_WSK(4, 0) MTD_WSK(6, 0) MTD_WSK(4, 6) MTD_WSK(6, 4) MTD_WSK(3, 4) MTD_WSK(3, 6)
    default: return nullptr;
    }
#undef MTD_WSK
}

}  // namespace

template <typename T> int walk_step_blocks(int LA, int LB, bool step_switch) {
    void *k = step_kernel<T>(LA, LB, step_switch);
    if (!k) return 0;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, kWalkBlock, 0) != cudaSuccess) return 0;
    return per * sms;
}

template <typename T>
cudaError_t launch_walk_step(int LA, int LB, bool step_switch, const WalkDesc<T> *d_desc, const WalkStepArgs &a,
                             int blocks, cudaStream_t st) {
    void *k = step_kernel<T>(LA, LB, step_switch);
    if (!k || blocks < 1) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(blocks);
    cfg.blockDim = dim3(kWalkBlock);
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&d_desc, (void *)&a};
    return cudaLaunchKernelExC(&cfg, k, args);
}

template int walk_step_blocks<float>(int, int, bool);
template int walk_step_blocks<double>(int, int, bool);
template cudaError_t launch_walk_step<float>(int, int, bool, const WalkDesc<float> *, const WalkStepArgs &, int,
                                             cudaStream_t);
template cudaError_t launch_walk_step<double>(int, int, bool, const WalkDesc<double> *, const WalkStepArgs &, int,
                                              cudaStream_t);

}  // namespace mtd
