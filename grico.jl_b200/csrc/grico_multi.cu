// Many right-hand sides at once: preconditioned CG run in lockstep on nrhs stacked systems
// (one operator apply with gridDim.y = nrhs per iteration, per-system scalars on the device,
// converged systems frozen), optionally as FP64 iterative refinement around FP32 inner solves
// (FP64 residuals and updates, FP32 operator applies).  Each system follows the reference's
// CG with its unpreconditioned stopping rule (solve.jl:376-431); the batching is this
// library's addition.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <vector>

#include "grico_host.h"
#include "grico_plan_internal.h"
#include "vector_kernels.cuh"

namespace grico {

int prepare_jacobi(GricoPlan* P, cudaStream_t st);

namespace {

constexpr int kMultiBlocks = 148;  // per system: partial sums [nrhs][kMultiBlocks]

// partial[s][blk] = sum a_s * b_s (or sum a_s * w * b_s with a weight vector shared by all systems)
template <typename T>
__global__ void multi_dot(const T* __restrict__ a, const T* __restrict__ b, const T* __restrict__ w, int64_t n,
                          double* __restrict__ partial) {
  __shared__ double sh[256];
  const int s = blockIdx.y;
  const T* as = a + int64_t(s) * n;
  const T* bs = b + int64_t(s) * n;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    acc += double(as[i]) * double(bs[i]) * (w ? double(w[i]) : 1.0);
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[int64_t(s) * gridDim.x + blockIdx.x] = sh[0];
}

// out[s] = sum_blk partial[s][blk]; one block per system
__global__ void multi_reduce(const double* __restrict__ partial, int blocks, double* __restrict__ out) {
  __shared__ double sh[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < blocks; i += blockDim.x) acc += partial[int64_t(blockIdx.x) * blocks + i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// x_s += alpha_s p_s ; r_s -= alpha_s q_s  for active systems with p.Ap > 0
template <typename T>
__global__ void multi_update(T* __restrict__ x, T* __restrict__ r, const T* __restrict__ p, const T* __restrict__ q,
                             const double* __restrict__ rz, const double* __restrict__ pap,
                             const int* __restrict__ active, int64_t n) {
  const int s = blockIdx.y;
  if (!active[s] || !(pap[s] > 0.0)) return;
  const T alpha = T(rz[s] / pap[s]);
  const int64_t o = int64_t(s) * n;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x) {
    x[o + i] += alpha * p[o + i];
    r[o + i] -= alpha * q[o + i];
  }
}

// z_s = dinv * r_s (dinv == nullptr: identity)
template <typename T>
__global__ void multi_precondition(const T* __restrict__ r, const T* __restrict__ dinv, T* __restrict__ z, int64_t n) {
  const int64_t o = int64_t(blockIdx.y) * n;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    z[o + i] = dinv ? dinv[i] * r[o + i] : r[o + i];
}

// p_s = z_s + (rz_new_s / rz_s) p_s ; rz_s = rz_new_s (active systems)
template <typename T>
__global__ void multi_direction(T* __restrict__ p, const T* __restrict__ z, const double* __restrict__ rz_new,
                                const double* __restrict__ rz, const int* __restrict__ active, int64_t n) {
  const int s = blockIdx.y;
  if (!active[s]) return;
  const T beta = T(rz_new[s] / rz[s]);
  const int64_t o = int64_t(s) * n;
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    p[o + i] = z[o + i] + beta * p[o + i];
}

__global__ void copy_scalars(double* __restrict__ dst, const double* __restrict__ src, const int* __restrict__ active,
                             int nrhs) {
  for (int s = threadIdx.x; s < nrhs; s += blockDim.x)
    if (active[s]) dst[s] = src[s];
}

// End of a lockstep iteration: count it for every active system and freeze the systems that met
// ||r||^2 <= tol2 or broke down (the stopping test of solve.jl:407-421 and the direction check
// of :414-416), on the device, so that several iterations run between two host reads.
// last_rr keeps the squared residual norm of the last iteration that ended finite and with a
// positive direction: after a breakdown (p.Ap <= 0) the update used alpha = r.z / p.Ap and rr no
// longer describes a valid iterate, so the report keeps the value before it
__global__ void multi_check(const double* __restrict__ pap, const double* __restrict__ rr,
                            const double* __restrict__ tol2, int* __restrict__ active, int* __restrict__ iters,
                            int* __restrict__ status, double* __restrict__ last_rr, int nrhs) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nrhs || !active[s]) return;
  iters[s] += 1;
  const double a = pap[s];
  if (!(a > 0.0)) {
    status[s] = isfinite(a) ? GRICO_ERR_BREAKDOWN : GRICO_ERR_NONFINITE;
    active[s] = 0;
    return;
  }
  const double v = rr[s];
  if (!isfinite(v)) {
    status[s] = GRICO_ERR_NONFINITE;
    active[s] = 0;
    return;
  }
  last_rr[s] = v;
  if (v <= tol2[s]) active[s] = 0;
}

template <typename S, typename D>
__global__ void cast_copy(const S* __restrict__ x, D* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] = D(x[i]);
}

// y += D(x)
template <typename S, typename D>
__global__ void cast_add(const S* __restrict__ x, D* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
    y[i] += D(x[i]);
}

int gblocks(int64_t n) { return int(std::min<int64_t>((n + 255) / 256, kMultiBlocks)); }

}  // namespace
}  // namespace grico

namespace grico {
namespace {

struct MultiResult {
  std::vector<int> iters, status;
  std::vector<double> rr;
};

// Work buffer `slot` of the plan's lockstep solver, `count` elements of T: kept on the plan and
// reallocated only to grow, so repeated solves on a plan allocate nothing (nullptr on failure).
// Slots 0-9: multi_cg; 10-18: grico_cg_solve_multi.
template <typename T>
T* solver_ws(GricoPlan* P, int slot, int64_t count) {
  DevBuf& b = P->solver_ws[slot];
  const size_t bytes = sizeof(T) * size_t(std::max<int64_t>(count, 1));
  if ((b.bytes < bytes || !b.ptr) && !b.alloc(bytes)) return nullptr;
  return b.get<T>();
}

// Lockstep preconditioned CG on nrhs stacked systems A x_s = b_s from x_s = 0, stopping
// system s once ||r_s||^2 <= tol2[s].  keep (optional): the instantiated iteration graph of an
// earlier call with the same x, dinv and nrhs on this plan (its other buffers are the plan's
// work vectors), reused instead of a new capture; a newly captured graph is left there for the
// caller to destroy.
template <typename T>
int multi_cg(GricoPlan* P, const T* b, T* x, int nrhs, const std::vector<double>& tol2, int maxiter, const T* dinv,
             bool graph, cudaStream_t st, MultiResult& res, cudaGraphExec_t* keep = nullptr) {
  const int64_t n = P->n_red;
  const int64_t nn = n * nrhs;
  T *r = solver_ws<T>(P, 0, nn), *z = solver_ws<T>(P, 1, nn), *p = solver_ws<T>(P, 2, nn), *q = solver_ws<T>(P, 3, nn);
  double* rz = solver_ws<double>(P, 4, 5 * int64_t(nrhs));
  double* partial = solver_ws<double>(P, 5, int64_t(nrhs) * kMultiBlocks);
  int* active = solver_ws<int>(P, 6, nrhs);
  double* tolb = solver_ws<double>(P, 7, nrhs);
  int* d_iters = solver_ws<int>(P, 8, nrhs);
  int* d_status = solver_ws<int>(P, 9, nrhs);
  if (!r || !z || !p || !q || !rz || !partial || !active || !tolb || !d_iters || !d_status) return GRICO_ERR_CUDA;
  double* rz_new = rz + nrhs;
  double* pap = rz + 2 * nrhs;
  double* rr = rz + 3 * nrhs;
  double* last_rr = rz + 4 * nrhs;
  const dim3 vg(gblocks(n), nrhs);
  auto dot = [&](const T* a, const T* c, double* out, cudaStream_t s) {
    multi_dot<T><<<dim3(kMultiBlocks, nrhs), 256, 0, s>>>(a, c, nullptr, n, partial);
    multi_reduce<<<nrhs, 256, 0, s>>>(partial, kMultiBlocks, out);
  };
  cudaMemsetAsync(x, 0, sizeof(T) * nn, st);
  cudaMemcpyAsync(r, b, sizeof(T) * nn, cudaMemcpyDeviceToDevice, st);
  multi_precondition<T><<<vg, 256, 0, st>>>(r, dinv, z, n);
  cudaMemcpyAsync(p, z, sizeof(T) * nn, cudaMemcpyDeviceToDevice, st);
  dot(r, z, rz, st);
  dot(r, r, rr, st);
  cudaMemcpyAsync(last_rr, rr, sizeof(double) * nrhs, cudaMemcpyDeviceToDevice, st);
  std::vector<double> h(2 * nrhs);
  std::vector<int> ha(nrhs, 1);
  cudaMemcpyAsync(h.data() + nrhs, rr, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  res.iters.assign(nrhs, 0);
  res.status.assign(nrhs, GRICO_OK);
  res.rr.assign(h.begin() + nrhs, h.end());
  int n_active = 0;
  for (int s = 0; s < nrhs; ++s) {
    ha[s] = res.rr[s] > tol2[s] ? 1 : 0;
    n_active += ha[s];
  }
  cudaMemcpyAsync(active, ha.data(), sizeof(int) * nrhs, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(tolb, tol2.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(d_iters, 0, sizeof(int) * nrhs, st);
  cudaMemsetAsync(d_status, 0, sizeof(int) * nrhs, st);  // GRICO_OK
  auto iteration = [&](cudaStream_t s) -> int {
    int rc = run_apply<T>(P, true, p, q, nrhs, s);
    if (rc) return rc;
    dot(p, q, pap, s);
    multi_update<T><<<vg, 256, 0, s>>>(x, r, p, q, rz, pap, active, n);
    dot(r, r, rr, s);
    multi_precondition<T><<<vg, 256, 0, s>>>(r, dinv, z, n);
    dot(r, z, rz_new, s);
    multi_direction<T><<<vg, 256, 0, s>>>(p, z, rz_new, rz, active, n);
    copy_scalars<<<1, 64, 0, s>>>(rz, rz_new, active, nrhs);
    multi_check<<<(nrhs + 63) / 64, 64, 0, s>>>(pap, rr, tolb, active, d_iters, d_status, last_rr,
                                                 nrhs);
    return GRICO_OK;
  };
  cudaGraphExec_t exec = keep ? *keep : nullptr;
  if (graph && n_active > 0 && !exec) {
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int crc = iteration(st);
      const cudaError_t ec = cudaStreamEndCapture(st, &g);
      if (crc == GRICO_OK && ec == cudaSuccess && g && cudaGraphInstantiate(&exec, g, 0) != cudaSuccess) exec = nullptr;
      if (g) cudaGraphDestroy(g);
    }
    (void)cudaGetLastError();
  }
  // The device freezes converged systems itself (multi_check), so the host reads the flags only
  // after a burst of iterations; a burst past the last convergence costs a few frozen
  // iterations, never a changed result.
  constexpr int kBurst = 8;
  int rc = GRICO_OK;
  std::vector<double> hrr(nrhs);
  for (int it = 0; it < maxiter && n_active > 0;) {
    const int k = std::min(kBurst, maxiter - it);
    for (int j = 0; j < k && rc == GRICO_OK; ++j) {
      if (exec) {
        if (cudaGraphLaunch(exec, st) != cudaSuccess) rc = GRICO_ERR_CUDA;
      } else {
        rc = iteration(st);
      }
    }
    if (rc != GRICO_OK) break;
    it += k;
    cudaMemcpyAsync(ha.data(), active, sizeof(int) * nrhs, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    n_active = 0;
    for (int s = 0; s < nrhs; ++s) n_active += ha[s];
  }
  if (keep) *keep = exec;
  else if (exec) cudaGraphExecDestroy(exec);
  cudaMemcpyAsync(res.iters.data(), d_iters, sizeof(int) * nrhs, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(res.status.data(), d_status, sizeof(int) * nrhs, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(hrr.data(), last_rr, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(ha.data(), active, sizeof(int) * nrhs, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  for (int s = 0; s < nrhs; ++s)
    if (res.iters[s] > 0) res.rr[s] = hrr[s];
  for (int s = 0; s < nrhs; ++s)
    if (ha[s] && res.status[s] == GRICO_OK) res.status[s] = GRICO_ERR_NOT_CONVERGED;
  if (!cuda_ok(cudaStreamSynchronize(st), "multi cg")) return GRICO_ERR_CUDA;
  return rc;
}

}  // namespace
}  // namespace grico

using namespace grico;

extern "C" int grico_cg_solve_multi(GricoPlan* P, const double* B, double* X, int nrhs, const GricoSolveOptions* opts,
                                    GricoSolveReport* reports, int flags) {
  if (!P || !B || !X || !opts || nrhs < 1 || nrhs > 65535) { set_error("cg multi: invalid argument"); return GRICO_ERR_INVALID; }
  if (opts->preconditioner != GRICO_PRECOND_IDENTITY && opts->preconditioner != GRICO_PRECOND_JACOBI) {
    set_error("cg multi: identity or Jacobi preconditioning");
    return GRICO_ERR_UNSUPPORTED_FORM;
  }
  if (opts->maxiter < 1 || !(opts->relative_tolerance >= 0) || !(opts->absolute_tolerance >= 0)) {
    set_error("cg multi: invalid options");
    return GRICO_ERR_INVALID;
  }
  if (P->n_red == 0) {  // every dof fixed: solved before the first iteration
    if (reports)
      for (int r = 0; r < nrhs; ++r) reports[r] = GricoSolveReport{};
    return GRICO_OK;
  }
  cudaStream_t st = P->stream;
  const int64_t n = P->n_red;
  const int64_t nn = n * nrhs;
  const bool graph = !(flags & GRICO_FLAG_NO_GRAPH);
  const bool mixed = (flags & GRICO_FLAG_MIXED) != 0;
  const double* bd = B;
  double* xd = X;
  if (flags & GRICO_FLAG_HOST_POINTERS) {
    double* bs = solver_ws<double>(P, 10, nn);
    xd = solver_ws<double>(P, 11, nn);
    if (!bs || !xd) return GRICO_ERR_CUDA;
    cudaMemcpyAsync(bs, B, sizeof(double) * nn, cudaMemcpyHostToDevice, st);
    bd = bs;
  }
  const double* dinv = nullptr;
  if (opts->preconditioner == GRICO_PRECOND_JACOBI) {
    if (int rc = prepare_jacobi(P, st)) return rc;
    dinv = P->w_dinv.get<double>();
  }
  // tolerances from ||b_s||
  double* part = solver_ws<double>(P, 12, int64_t(nrhs) * kMultiBlocks);
  double* bn = solver_ws<double>(P, 13, nrhs);
  if (!part || !bn) return GRICO_ERR_CUDA;
  multi_dot<double><<<dim3(kMultiBlocks, nrhs), 256, 0, st>>>(bd, bd, nullptr, n, part);
  multi_reduce<<<nrhs, 256, 0, st>>>(part, kMultiBlocks, bn);
  std::vector<double> bnorm2(nrhs), tol2(nrhs);
  cudaMemcpyAsync(bnorm2.data(), bn, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  for (int s = 0; s < nrhs; ++s) {
    const double t = std::max(opts->absolute_tolerance, opts->relative_tolerance * std::sqrt(bnorm2[s]));
    tol2[s] = t * t;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  MultiResult res;
  int rc = GRICO_OK;
  std::vector<int> total(nrhs, 0), status(nrhs, GRICO_OK);
  std::vector<double> final_rr(nrhs, 0.0);
  if (!mixed) {
    rc = multi_cg<double>(P, bd, xd, nrhs, tol2, opts->maxiter, dinv, graph, st, res);
    total = res.iters;
    status = res.status;
    final_rr = res.rr;
  } else {
    // FP64 iterative refinement: r = b - A x in FP64, FP32 inner CG on A e = r to 1e-4
    // relative, x += e; repeat until every system meets its FP64 tolerance.
    double* r64 = solver_ws<double>(P, 14, nn);
    float* r32 = solver_ws<float>(P, 15, nn);
    float* e32 = solver_ws<float>(P, 16, nn);
    double* ax = solver_ws<double>(P, 17, nn);
    float* dinv32 = dinv ? solver_ws<float>(P, 18, n) : nullptr;
    if (!r64 || !r32 || !e32 || !ax || (dinv && !dinv32)) return GRICO_ERR_CUDA;
    if (dinv) cast_copy<double, float><<<gblocks(n), 256, 0, st>>>(dinv, dinv32, n);
    cudaMemsetAsync(xd, 0, sizeof(double) * nn, st);
    cudaMemcpyAsync(r64, bd, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
    std::vector<int> done(nrhs, 0);
    cudaGraphExec_t inner_graph = nullptr;
    for (int outer = 0; outer < 60; ++outer) {
      multi_dot<double><<<dim3(kMultiBlocks, nrhs), 256, 0, st>>>(r64, r64, nullptr, n, part);
      multi_reduce<<<nrhs, 256, 0, st>>>(part, kMultiBlocks, bn);
      cudaMemcpyAsync(final_rr.data(), bn, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st);
      cudaStreamSynchronize(st);
      bool all = true;
      std::vector<double> inner_tol2(nrhs);
      for (int s = 0; s < nrhs; ++s) {
        done[s] = final_rr[s] <= tol2[s] || status[s] != GRICO_OK;
        all = all && done[s];
        // converged systems get an unreachable inner tolerance of 0 but a zero residual
        inner_tol2[s] = done[s] ? 1e300 : 1e-8 * final_rr[s];
      }
      if (all) break;
      bool over = false;
      for (int s = 0; s < nrhs; ++s) over = over || (!done[s] && total[s] >= opts->maxiter);
      if (over) break;
      cast_copy<double, float><<<gblocks(nn), 256, 0, st>>>(r64, r32, nn);
      // every refinement step solves into the same buffers: one iteration graph serves them all
      rc = multi_cg<float>(P, r32, e32, nrhs, inner_tol2, opts->maxiter, dinv32, graph, st, res, &inner_graph);
      if (rc) break;
      for (int s = 0; s < nrhs; ++s) {
        if (done[s]) continue;
        total[s] += res.iters[s];
        if (res.status[s] != GRICO_OK && res.status[s] != GRICO_ERR_NOT_CONVERGED) status[s] = res.status[s];
      }
      cast_add<float, double><<<gblocks(nn), 256, 0, st>>>(e32, xd, nn);
      cudaMemcpyAsync(r64, bd, sizeof(double) * nn, cudaMemcpyDeviceToDevice, st);
      run_apply<double>(P, true, xd, ax, nrhs, st);
      axpby_kernel<double><<<grid_blocks(nn), 256, 0, st>>>(-1.0, ax, 1.0, r64, nn);
    }
    if (inner_graph) cudaGraphExecDestroy(inner_graph);
    for (int s = 0; s < nrhs; ++s)
      if (status[s] == GRICO_OK && final_rr[s] > tol2[s]) status[s] = GRICO_ERR_NOT_CONVERGED;
  }
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (flags & GRICO_FLAG_HOST_POINTERS) cudaMemcpyAsync(X, xd, sizeof(double) * nn, cudaMemcpyDeviceToHost, st);
  if (!cuda_ok(cudaStreamSynchronize(st), "cg multi")) return GRICO_ERR_CUDA;
  int worst = rc;
  for (int s = 0; s < nrhs; ++s) {
    if (reports) {
      reports[s].iterations = total[s];
      reports[s].status = status[s];
      reports[s].initial_residual = std::sqrt(bnorm2[s]);
      reports[s].final_residual = std::sqrt(final_rr[s]);
      reports[s].seconds = ms * 1e-3;
    }
    if (!worst && status[s]) worst = status[s];
  }
  if (worst == GRICO_ERR_NOT_CONVERGED) set_error("cg multi: a system did not converge in maxiter iterations");
  return worst;
}
