// Internal interface of the device multigrid used by the Krylov drivers.
#pragma once
#include <cuda_runtime.h>

#include "grico_plan_internal.h"

namespace grico {
// z = V-cycle(r) on the finest level of mg, on stream st (multigrid.jl:858-889)
int mg_vcycle_device(GricoMultigrid* mg, const double* r, double* z, cudaStream_t st);
// GRICO_SMOOTHER_* of mg
int mg_smoother(const GricoMultigrid* mg);
// identity of mg's current V-cycle: unique per multigrid object, renewed when the cycle changes
uint64_t mg_identity(const GricoMultigrid* mg);
// sum of the level plans' epochs (changes when a level's kernels or their arguments change)
uint64_t mg_epoch(const GricoMultigrid* mg);
// tensor-core convolution (csrc/grico_cnn.cu): packed BF16 weights from FP32 [Co][Ci][27], and
// the forward pass on channels-last BF16 activations (out_cf: FP32 channel-first output)
int conv_tc_pack(const float* w, int Ci, int Co, void* wp, cudaStream_t st);
int conv_tc_forward(const void* x, const void* wp, const float* bias, void* y, int out_cf, int B, int Ci, int Co,
                    int Z, int Y, int X, int relu, cudaStream_t st);
}  // namespace grico
