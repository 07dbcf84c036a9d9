// Building blocks of the sharded reduced solve: one rank owns a contiguous range of cells, its
// local reduced vector holds the dofs it owns first and the ghost dofs it shares after them.
// The partition-surface sum of an apply is a pack into a halo buffer indexed by global halo
// slot, a sum over ranks (the caller's collective), and an unpack.  The CG steps read their
// scalars from device memory, so a rank sums them with one collective and no host round trip;
// every reduction covers the owned prefix only, so the sum over ranks counts each dof once.
// (The reference has one shared-memory process: solve.jl:376-431 is the unsharded loop.)
#include <cuda_runtime.h>

#include <algorithm>

#include "grico_host.h"
#include "grico_plan_internal.h"
#include "vector_kernels.cuh"

namespace grico {
namespace {

__global__ void halo_pack(const double* __restrict__ y, const int32_t* __restrict__ local,
                          const int32_t* __restrict__ slot, int64_t n, double* __restrict__ buf) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    buf[slot[i]] = y[local[i]];
}

__global__ void halo_unpack(double* __restrict__ y, const int32_t* __restrict__ local,
                            const int32_t* __restrict__ slot, int64_t n, const double* __restrict__ buf) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[local[i]] = buf[slot[i]];
}

// x += alpha p, r -= alpha q on n entries with alpha = s[0] / s[1]; partial sums of r*r over
// the first n_sum entries
__global__ void shard_update_xr(double* __restrict__ x, double* __restrict__ r, const double* __restrict__ p,
                                const double* __restrict__ q, const double* __restrict__ s, int64_t n, int64_t n_sum,
                                double* __restrict__ partial) {
  __shared__ double sh[32];
  const bool ok = s[1] > 0.0;  // breakdown: keep x and r, the host reports it
  const double alpha = ok ? s[0] / s[1] : 0.0;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    double ri = r[i];
    if (ok) {
      x[i] += alpha * p[i];
      ri -= alpha * q[i];
      r[i] = ri;
    }
    if (i < n_sum) acc += ri * ri;
  }
  acc = block_sum<double>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// z = dinv .* r (dinv == nullptr: z = r); partial sums of r*z over the first n_sum entries
__global__ void shard_precondition(const double* __restrict__ dinv, const double* __restrict__ r,
                                   double* __restrict__ z, int64_t n, int64_t n_sum, double* __restrict__ partial) {
  __shared__ double sh[32];
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    const double zi = dinv ? dinv[i] * r[i] : r[i];
    z[i] = zi;
    if (i < n_sum) acc += r[i] * zi;
  }
  acc = block_sum<double>(acc, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = acc;
}

// p = z + (s[3] / s[0]) p; s[0] = s[3] follows as a second launch, after every block has
// read s[0]
__global__ void shard_direction(double* __restrict__ p, const double* __restrict__ z, const double* __restrict__ s,
                                int64_t n) {
  const double beta = s[3] / s[0];
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

__global__ void shard_roll(double* __restrict__ s) { s[0] = s[3]; }

int blocks_for(int64_t n) { return int(std::min<int64_t>((n + 255) / 256, kRedBlocks)); }

bool valid_n(int64_t n, const char* what) {
  if (n < 0) {
    set_error(std::string(what) + ": negative length");
    return false;
  }
  return true;
}

int launch_status(const char* what) { return cuda_ok(cudaGetLastError(), what) ? GRICO_OK : GRICO_ERR_CUDA; }

}  // namespace
}  // namespace grico

using namespace grico;

extern "C" {

int grico_halo_pack(const double* y, const int32_t* local, const int32_t* slot, int64_t n, double* buf,
                    int64_t n_slots, void* stream) {
  if (!valid_n(n, "halo pack") || !valid_n(n_slots, "halo pack")) return GRICO_ERR_INVALID;
  if (n_slots > 0 && !buf) { set_error("halo pack: buffer missing"); return GRICO_ERR_INVALID; }
  if (n > 0 && (!y || !local || !slot)) { set_error("halo pack: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n_slots > 0) cudaMemsetAsync(buf, 0, sizeof(double) * size_t(n_slots), st);
  if (n > 0) halo_pack<<<blocks_for(n), 256, 0, st>>>(y, local, slot, n, buf);
  return launch_status("halo pack");
}

int grico_halo_unpack(double* y, const int32_t* local, const int32_t* slot, int64_t n, const double* buf,
                      void* stream) {
  if (!valid_n(n, "halo unpack")) return GRICO_ERR_INVALID;
  if (n == 0) return GRICO_OK;
  if (!y || !local || !slot || !buf) { set_error("halo unpack: invalid argument"); return GRICO_ERR_INVALID; }
  halo_unpack<<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(y, local, slot, n, buf);
  return launch_status("halo unpack");
}

int grico_vec_dot(int64_t n, const double* x, const double* y, double* out, double* partial, void* stream) {
  if (!valid_n(n, "dot")) return GRICO_ERR_INVALID;
  if (!out || !partial || (n > 0 && (!x || !y))) { set_error("dot: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dot_partial<double><<<kRedBlocks, kRedThreads, 0, st>>>(x, y, n, partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, out);
  return launch_status("dot");
}

int grico_vec_axpby(int64_t n, double a, const double* x, double b, double* y, void* stream) {
  if (!valid_n(n, "axpby")) return GRICO_ERR_INVALID;
  if (n == 0) return GRICO_OK;
  if (!x || !y) { set_error("axpby: invalid argument"); return GRICO_ERR_INVALID; }
  axpby_kernel<double><<<blocks_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(a, x, b, y, n);
  return launch_status("axpby");
}

int grico_vec_invert(int64_t n, const double* d, double* dinv, void* stream) {
  if (!valid_n(n, "invert")) return GRICO_ERR_INVALID;
  if (n == 0) return GRICO_OK;
  if (!d || !dinv) { set_error("invert: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  DevBuf flag;
  if (!flag.alloc(sizeof(int))) return GRICO_ERR_CUDA;
  cudaMemsetAsync(flag.ptr, 0, sizeof(int), st);
  invert_diagonal<<<blocks_for(n), 256, 0, st>>>(d, dinv, n, flag.get<int>());
  int bad = 0;
  cudaMemcpyAsync(&bad, flag.ptr, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "invert")) return GRICO_ERR_CUDA;
  if (bad) {
    set_error("Jacobi preconditioner found a zero or non-finite diagonal entry");  // solve.jl:740-748
    return GRICO_ERR_NONFINITE;
  }
  return GRICO_OK;
}

int grico_cg_update_xr(int64_t n, int64_t n_sum, double* x, double* r, const double* p, const double* q,
                       double* scalars, double* partial, void* stream) {
  if (!valid_n(n, "cg update") || n_sum < 0 || n_sum > n) { set_error("cg update: invalid lengths"); return GRICO_ERR_INVALID; }
  if (!scalars || !partial || (n > 0 && (!x || !r || !p || !q))) { set_error("cg update: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  shard_update_xr<<<kRedBlocks, kRedThreads, 0, st>>>(x, r, p, q, scalars, n, n_sum, partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, scalars + 2);
  return launch_status("cg update");
}

int grico_cg_precondition(int64_t n, int64_t n_sum, const double* dinv, const double* r, double* z, double* scalars,
                          double* partial, void* stream) {
  if (!valid_n(n, "cg precondition") || n_sum < 0 || n_sum > n) { set_error("cg precondition: invalid lengths"); return GRICO_ERR_INVALID; }
  if (!scalars || !partial || (n > 0 && (!r || !z))) { set_error("cg precondition: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  shard_precondition<<<kRedBlocks, kRedThreads, 0, st>>>(dinv, r, z, n, n_sum, partial);
  reduce_final<<<1, kRedThreads, 0, st>>>(partial, kRedBlocks, scalars + 3);
  return launch_status("cg precondition");
}

int grico_cg_direction(int64_t n, double* p, const double* z, double* scalars, void* stream) {
  if (!valid_n(n, "cg direction")) return GRICO_ERR_INVALID;
  if (!scalars || (n > 0 && (!p || !z))) { set_error("cg direction: invalid argument"); return GRICO_ERR_INVALID; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (n > 0) shard_direction<<<blocks_for(n), 256, 0, st>>>(p, z, scalars, n);
  shard_roll<<<1, 1, 0, st>>>(scalars);
  return launch_status("cg direction");
}

}  // extern "C"
