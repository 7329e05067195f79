// nnbias.h -- the learned-bias object as used from a context's step.
#pragma once

#include <cuda_runtime.h>

#include "../../include/metad_b200.h"

namespace mtd {

// V and dV/ds at the device point d_s (D doubles) into d_vdv = [V, dV[0..D)],
// enqueued on st: with nn, the network plus the exact FP64 sum over the hills
// [h_from, nh) deposited since it was fitted; without, the exact sum over all
// hills.
mtd_status nnbias_enqueue_vdv(mtd_nnbias *nb, const double *d_s, double *d_vdv, bool nn, int h_from,
                              cudaStream_t st);

}  // namespace mtd
