// Internal interface of the device multigrid used by the Krylov drivers.
#pragma once
#include <cuda_runtime.h>

#include "grico_plan_internal.h"

namespace grico {
// z = V-cycle(r) on the finest level of mg, on stream st (multigrid.jl:858-889)
int mg_vcycle_device(GricoMultigrid* mg, const double* r, double* z, cudaStream_t st);
// GRICO_SMOOTHER_* of mg
int mg_smoother(const GricoMultigrid* mg);
}  // namespace grico
